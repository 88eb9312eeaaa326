// capi.cu -- the extern "C" boundary of libymgpu (declared in include/ymgpu.h).
//
// Host-side mirror of the reference crate's lattice/ensemble entry points:
// validation follows the reference's fail-closed checks in the same order
// and reports the same variants (include/ym_status.h); device work is
// enqueued on the handle's stream and synchronised before results return.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "ym_internal.hpp"

using ym::ChainInfo;
using ym::Tile;

namespace {

thread_local int g_last_cuda_error = 0;

int32_t cuda_status(cudaError_t err) {
    if (err == cudaSuccess) return YM_OK;
    g_last_cuda_error = (int)err;
    return YM_ERR_CUDA;
}

}  // namespace

int32_t ym::record_cuda_status(cudaError_t err) { return cuda_status(err); }

// ---- device memory -----------------------------------------------------
// Every device buffer of the library comes from the device's stream-ordered
// memory pool, allocated and freed on one allocation stream per device, with
// the pool's release threshold raised so that freed blocks stay in the pool
// for the next handle instead of going back to the driver.  Plain
// cudaMalloc / cudaFree on these machines take milliseconds each and, about
// one call in forty, 50 to 180 ms, which a batch of short campaigns (each
// creating and destroying handles) would otherwise pay many times.
// dev_alloc synchronises the allocation stream, so a block is ready for any
// stream when it returns; dev_free first waits for the device to go idle, as
// cudaFree does, so no kernel in flight on any stream still reads the block.
// The pool keeps what it holds until the process exits; an allocation that
// finds the device full gives the pool's idle blocks back and tries once
// more.
namespace {

struct DevicePool {
    std::mutex lock;
    cudaStream_t stream[64] = {};
};

DevicePool &device_pool() {
    static DevicePool p;
    return p;
}

cudaError_t alloc_stream(int dev, cudaStream_t *out) {
    DevicePool &p = device_pool();
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(p.lock);
    if (!p.stream[dev]) {
        cudaMemPool_t pool = nullptr;
        cudaError_t err = cudaDeviceGetDefaultMemPool(&pool, dev);
        uint64_t keep = UINT64_MAX;
        if (err == cudaSuccess) err = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&p.stream[dev], cudaStreamNonBlocking);
        if (err != cudaSuccess) return err;
    }
    *out = p.stream[dev];
    return cudaSuccess;
}

}  // namespace

cudaError_t ym::dev_alloc(void **ptr, size_t bytes) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    cudaStream_t s = nullptr;
    if (err == cudaSuccess) err = alloc_stream(dev, &s);
    if (err == cudaSuccess) {
        err = cudaMallocAsync(ptr, bytes, s);
        if (err == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            cudaMemPool_t pool = nullptr;
            if (cudaStreamSynchronize(s) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
                cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
                err = cudaMallocAsync(ptr, bytes, s);
        }
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    return err;
}

void ym::dev_free(void *ptr) {
    if (!ptr) return;
    cudaPointerAttributes at{};
    cudaStream_t s = nullptr;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || alloc_stream(at.device, &s) != cudaSuccess) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != at.device) cudaSetDevice(at.device);
    cudaDeviceSynchronize();
    cudaFreeAsync(ptr, s);
    if (cur != at.device) cudaSetDevice(cur);
}

namespace {

#define YM_CUDA(call)                                 \
    do {                                              \
        cudaError_t err__ = (call);                   \
        if (err__ != cudaSuccess) return cuda_status(err__); \
    } while (0)

constexpr int64_t kMaxSu3Links = int64_t(1) << 18;   // su3_lattice.rs:17
constexpr int64_t kMaxSu2Links = int64_t(1) << 20;   // lib.rs:21
constexpr double kMaxSu3Beta = 12.0;                 // su3_ensemble.rs:24
constexpr double kMaxSu2Beta = 8.0;                  // su2_ensemble.rs:18
constexpr double kMinAngle = 1.0e-8;                 // su3_ensemble.rs:27
constexpr double kMaxAngle = 1.0;                    // su3_ensemble.rs:28
constexpr double kLiftedMaxAngle = 2.5;              // two-row sweeps with the cap lifted
constexpr int kGraphSweeps = 8;                      // sweeps per captured graph

template <class T>
cudaError_t dalloc(T **p, size_t count) {
    return ym::dev_alloc(reinterpret_cast<void **>(p), count * sizeof(T) + 16);
}

void free_all(ym_ensemble *e) {
    if (e->sweep_graph) cudaGraphExecDestroy(e->sweep_graph);
    if (e->measure_graph) cudaGraphExecDestroy(e->measure_graph);
    if (e->run_graph) cudaGraphExecDestroy(e->run_graph);
    if (e->glueball_graph) cudaGraphExecDestroy(e->glueball_graph);
    if (e->su2_graph) cudaGraphExecDestroy(e->su2_graph);
    if (e->d_gb_series) ym::dev_free(e->d_gb_series);
    if (e->d_series) ym::dev_free(e->d_series);
    if (e->d_wilson_series) ym::dev_free(e->d_wilson_series);
    if (e->d_poly_series) ym::dev_free(e->d_poly_series);
    if (e->d_loop_row) ym::dev_free(e->d_loop_row);
    if (e->d_series_row) ym::dev_free(e->d_series_row);
    for (auto &pool : e->events)
        for (auto &p : pool) {
            cudaEventDestroy(p.start);
            cudaEventDestroy(p.stop);
        }
    void *ptrs[] = {e->d_chains, e->d_half_tiles, e->d_site_tiles, e->d_mixed_tiles, e->d_site_tile_first,
                    e->d_links, e->d_staging, e->d_partial, e->d_partial2, e->d_result,
                    e->d_result2, e->d_accepts, e->d_sweep, e->d_rng, e->d_ref_counts,
                    e->d_error, e->d_obs_partial, e->d_obs_out, e->d_site_vals,
                    e->d_slice_chain, e->d_slice_t, e->d_slice_plaq, e->d_slice_rect,
                    e->d_links_tmp, e->d_query_error, e->d_query, e->d_steps, e->d_terms,
                    e->d_tr_partial};
    for (void *p : ptrs)
        if (p) ym::dev_free(p);
    for (auto &l : e->layouts)
        if (l.d_items) ym::dev_free(l.d_items);
    for (auto &l : e->layouts)
        if (l.d_chain_ctas) ym::dev_free(l.d_chain_ctas);
    if (e->stream) cudaStreamDestroy(e->stream);
}

int32_t validate_angle(double a) {
    if (!std::isfinite(a) || a < kMinAngle || a > kMaxAngle)
        return YM_ERR_PROPOSAL_ANGLE_OUTSIDE_REFERENCE_RANGE;
    return YM_OK;
}

// The half width a handle's sweeps accept: the reference's [1e-8, 1], or up
// to kLiftedMaxAngle on a two-row handle whose angle cap was lifted.
int32_t validate_angle_for(const ym_ensemble *e, double a) {
    if (e->angle_cap_lifted && e->precision == YM_PREC_F32_TWO_ROW &&
        std::isfinite(a) && a > kMaxAngle && a <= kLiftedMaxAngle)
        return YM_OK;
    return validate_angle(a);
}

int32_t validate_su3_betas(const ym_ensemble *e) {
    for (const ChainInfo &c : e->chains)
        if (!std::isfinite(c.beta) || c.beta < 0.0 || c.beta > kMaxSu3Beta)
            return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    return YM_OK;
}

int32_t require_checkerboard(const ym_ensemble *e) {
    for (const ChainInfo &c : e->chains)
        for (int d = 0; d < 4; ++d)
            if (c.n[d] % 2) return YM_ERR_NOT_CHECKERBOARDABLE;
    return YM_OK;
}

int32_t set_device(const ym_ensemble *e) { return cuda_status(cudaSetDevice(e->device)); }

size_t reals_per_link(const ym_ensemble *e) { return e->group == YM_GROUP_SU3 ? 18 : 4; }

bool f32(const ym_ensemble *e) { return e->precision == YM_PREC_F32_TWO_ROW; }

cudaError_t identity(ym_ensemble *e) {
    if (f32(e)) return ym::launch_f32_identity(e);
    return e->group == YM_GROUP_SU3 ? ym::launch_su3_identity(e) : ym::launch_su2_identity(e);
}

cudaError_t from_aos(ym_ensemble *e, int64_t chain) {
    if (f32(e)) return ym::launch_f32_from_aos(e, chain);
    return e->group == YM_GROUP_SU3 ? ym::launch_su3_from_aos(e, chain) : ym::launch_su2_from_aos(e, chain);
}

cudaError_t to_aos(ym_ensemble *e, int64_t chain) {
    if (f32(e)) return ym::launch_f32_to_aos(e, chain);
    return e->group == YM_GROUP_SU3 ? ym::launch_su3_to_aos(e, chain) : ym::launch_su2_to_aos(e, chain);
}

// Kernels that read full binary64 SU(3) links.
int32_t require_su3_f64(const ym_ensemble *e) {
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    if (e->precision != YM_PREC_F64) return YM_ERR_UNSUPPORTED_PRECISION;
    return YM_OK;
}

// Reads and clears the device error bits of bounded loops that gave up.
int32_t take_device_error(ym_ensemble *e) {
    unsigned bits = 0;
    cudaError_t err = cudaMemcpyAsync(&bits, e->d_error, sizeof bits, cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return cuda_status(err);
    if (!bits) return YM_OK;
    err = cudaMemsetAsync(e->d_error, 0, sizeof(unsigned), e->stream);
    if (err != cudaSuccess) return cuda_status(err);
    if (bits & 1u) return YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED;
    if (bits & 16u) return YM_ERR_NON_FINITE_STAPLE;
    if (bits & 4u) return YM_ERR_ALGEBRA_PROJECTION_RESIDUAL;
    if (bits & 8u) return YM_ERR_NON_UNITARY_MATRIX;
    return YM_ERR_NON_FINITE_STATISTIC;
}

// Measurement scratch (allocated on first use, kept with the handle).
cudaError_t ensure_obs_scratch(ym_ensemble *e) {
    if (e->d_obs_partial) return cudaSuccess;
    int64_t sites = 0;
    std::vector<int32_t> sc, st;
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        sites += e->chains[ch].volume;
        for (int t = 0; t < e->chains[ch].n[3]; ++t) {
            sc.push_back((int32_t)ch);
            st.push_back(t);
        }
    }
    e->n_slices = (int64_t)sc.size();
    cudaError_t err = dalloc(&e->d_obs_partial, (size_t)e->n_site_tiles * 96);
    if (err == cudaSuccess) err = dalloc(&e->d_obs_out, (size_t)e->n_chains * 96);
    if (err == cudaSuccess) err = dalloc(&e->d_site_vals, (size_t)sites);
    if (err == cudaSuccess) err = dalloc(&e->d_slice_chain, sc.size());
    if (err == cudaSuccess) err = dalloc(&e->d_slice_t, st.size());
    if (err == cudaSuccess) err = dalloc(&e->d_slice_plaq, sc.size());
    if (err == cudaSuccess) err = dalloc(&e->d_slice_rect, sc.size());
    if (err == cudaSuccess)
        err = cudaMemcpy(e->d_slice_chain, sc.data(), sc.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (err == cudaSuccess)
        err = cudaMemcpy(e->d_slice_t, st.data(), st.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    return err;
}

bool same_geometry(const ym_ensemble *a, const ym_ensemble *b) {
    if (a->n_chains != b->n_chains || a->group != b->group || a->device != b->device ||
        a->precision != b->precision)
        return false;
    for (int64_t ch = 0; ch < a->n_chains; ++ch)
        for (int d = 0; d < 4; ++d)
            if (a->chains[ch].n[d] != b->chains[ch].n[d]) return false;
    return true;
}

// glueball_operators.rs:72-91 / glueball_smearing.rs:83-108 spatial checks.
int32_t require_cubic_spatial(const ym_ensemble *e, int min_extent) {
    for (const ChainInfo &c : e->chains) {
        for (int d = 0; d < 3; ++d)
            if (c.n[d] < min_extent) return YM_ERR_SPATIAL_EXTENT_TOO_SMALL;
        if (c.n[0] != c.n[1] || c.n[1] != c.n[2]) return YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC;
    }
    return YM_OK;
}

// Runs `launch` and, when profiling is on, brackets it with an event pair.
template <class F>
cudaError_t timed(ym_ensemble *e, int kernel, F launch) {
    if (!e->profiling) return launch();
    auto &pool = e->events[kernel];
    size_t &used = e->events_used[kernel];
    if (used == pool.size()) {
        ym_ensemble::EventPair p{};
        cudaError_t err = cudaEventCreate(&p.start);
        if (err == cudaSuccess) err = cudaEventCreate(&p.stop);
        if (err != cudaSuccess) return err;
        pool.push_back(p);
    }
    const ym_ensemble::EventPair &p = pool[used++];
    cudaError_t err = cudaEventRecord(p.start, e->stream);
    if (err == cudaSuccess) err = launch();
    if (err == cudaSuccess) err = cudaEventRecord(p.stop, e->stream);
    return err;
}

// Device time of run() on the handle's stream, in milliseconds.
template <class F>
cudaError_t time_on_stream(ym_ensemble *e, F run, float *ms) {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t err = cudaEventCreate(&a);
    if (err == cudaSuccess) err = cudaEventCreate(&b);
    if (err == cudaSuccess) err = cudaEventRecord(a, e->stream);
    if (err == cudaSuccess) err = run();
    if (err == cudaSuccess) err = cudaEventRecord(b, e->stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(b);
    if (err == cudaSuccess) err = cudaEventElapsedTime(ms, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    return err;
}

// The chain-resident path applies to SU(3) FP64 handles whose every chain
// fits one CTA's shared memory; profiled runs keep the tiled launches so
// each sub-sweep keeps its event pair.
bool resident_candidate(const ym_ensemble *e) {
    return e->group == YM_GROUP_SU3 && e->precision == YM_PREC_F64 && !e->profiling &&
           !e->fast_sweeps && e->resident_choice != 0 && ym::resident_fits(e);
}

constexpr int64_t kTuneSweeps = 4;   // sweeps timed per path when choosing
// Sweeps a call needs before the layout tuner runs: its probes (one warm
// sweep, then kTuneSweeps per layout, all ordinary sweeps of the chains
// launched without graph replay) are then at most half of the call.
constexpr int64_t kLayoutTuneMin = 2 * (ym::kSweepLayouts * kTuneSweeps + 1);

// Captured sweep graphs hold the launches of one layout and one form of the
// sub-sweep kernels; they are dropped when either changes.
void drop_sweep_graphs(ym_ensemble *e) {
    if (e->sweep_graph) cudaGraphExecDestroy(e->sweep_graph);
    e->sweep_graph = nullptr;
    if (e->measure_graph) cudaGraphExecDestroy(e->measure_graph);
    e->measure_graph = nullptr;
    if (e->run_graph) cudaGraphExecDestroy(e->run_graph);
    e->run_graph = nullptr;
}

// Selects sub-sweep layout li.
void set_layout(ym_ensemble *e, int32_t li) {
    if (e->sweep_layout == li && e->layout_tuned) return;
    e->sweep_layout = li;
    drop_sweep_graphs(e);
}

}  // namespace

extern "C" {

int32_t ym_last_cuda_error(void) { return g_last_cuda_error; }

int32_t ym_device_release_pooled_memory(int32_t device) {
    int count = 0, current = 0;
    YM_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return YM_ERR_INVALID_ARGUMENT;
    YM_CUDA(cudaGetDevice(&current));
    // the caller's current device is restored whatever happens
    cudaError_t err = cudaSetDevice(device);
    if (err == cudaSuccess) err = cudaDeviceSynchronize();
    cudaMemPool_t pool = nullptr;
    if (err == cudaSuccess) err = cudaDeviceGetDefaultMemPool(&pool, device);
    if (err == cudaSuccess) err = cudaMemPoolTrimTo(pool, 0);
    const cudaError_t back = cudaSetDevice(current);
    YM_CUDA(err);
    YM_CUDA(back);
    return YM_OK;
}

int32_t ym_ensemble_create(const ym_ensemble_desc *desc, ym_ensemble **out) {
    if (!desc || !out || !desc->extents || !desc->beta || !desc->chain_seed) return YM_ERR_NULL_ARGUMENT;
    *out = nullptr;
    if (desc->n_chains < 1 || desc->n_chains > (int64_t(1) << 30)) return YM_ERR_INVALID_ARGUMENT;
    if (desc->group != YM_GROUP_SU3 && desc->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    if (desc->precision != YM_PREC_F64 &&
        !(desc->precision == YM_PREC_F32_TWO_ROW && desc->group == YM_GROUP_SU3))
        return YM_ERR_UNSUPPORTED_PRECISION;

    ym_ensemble *e = new (std::nothrow) ym_ensemble();
    if (!e) return YM_ERR_ALLOCATION_FAILED;
    e->group = desc->group;
    e->precision = desc->precision;
    e->device = desc->device;
    e->n_chains = desc->n_chains;
    // storage elements per link: double2 (FP64 SU(3): 9, SU(2): 2) or float2
    // (two-row binary32 SU(3): 6); chain offsets count those elements
    const int64_t per_link = e->precision == YM_PREC_F32_TWO_ROW ? 6 : (e->group == YM_GROUP_SU3 ? 9 : 2);

    // Lattice4::new_identity / Su3Lattice4::new_identity checks
    // (lib.rs:242-263, su3_lattice.rs:85-106), per chain.
    int64_t offset = 0;
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        const int64_t *n = desc->extents + 4 * ch;
        ChainInfo c{};
        int64_t sites = 1;
        for (int d = 0; d < 4; ++d) {
            if (n[d] < 2) { delete e; return YM_ERR_INVALID_LATTICE_EXTENT; }
        }
        for (int d = 0; d < 4; ++d) {
            if (n[d] > (int64_t(1) << 30) || sites > INT64_MAX / n[d]) { delete e; return YM_ERR_LATTICE_SIZE_OVERFLOW; }
            sites *= n[d];
            c.n[d] = (int32_t)n[d];
        }
        if (sites > INT64_MAX / 4) { delete e; return YM_ERR_LATTICE_SIZE_OVERFLOW; }
        const int64_t links = sites * 4;
        const int64_t cap = e->group == YM_GROUP_SU3 ? kMaxSu3Links : kMaxSu2Links;
        if (!desc->lift_reference_caps && links > cap) { delete e; return YM_ERR_LATTICE_TOO_LARGE; }
        c.eo = (n[3] % 2 == 0) ? 1 : 0;
        c.volume = sites;
        c.half = c.eo ? sites / 2 : sites;
        c.offset = offset;
        c.beta = desc->beta[ch];
        c.seed = desc->chain_seed[ch];
        offset += 4 * per_link * sites;
        e->chains.push_back(c);
        e->chain_links.push_back(links);
        e->total_links += links;
        if (links > e->max_chain_links) e->max_chain_links = links;
    }
    // total_elems counts 16-byte units of link storage
    e->total_elems = e->precision == YM_PREC_F32_TWO_ROW ? (offset + 1) / 2 : offset;
    e->proposals.assign((size_t)e->n_chains, 0);

    // Work tiles: sub-sweeps cover the checkerboard half of every chain,
    // measurements cover every site; a tile never straddles two chains.
    std::vector<Tile> half, site;
    std::vector<int32_t> first;
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        const ChainInfo &c = e->chains[ch];
        for (int64_t s = 0; s < c.half; s += ym::kSweepThreads) half.push_back(Tile{(int32_t)ch, 0, s});
        first.push_back((int32_t)site.size());
        for (int64_t s = 0; s < c.volume; s += ym::kSiteThreads) site.push_back(Tile{(int32_t)ch, 0, s});
    }
    first.push_back((int32_t)site.size());
    // even tile k of a chain next to its odd tile k, so both parities of a
    // region are in flight (and in L2) together
    std::vector<Tile> mixed;
    mixed.reserve(site.size());
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        const ChainInfo &c = e->chains[ch];
        std::vector<Tile> ev, od;
        for (int32_t t = first[(size_t)ch]; t < first[(size_t)ch + 1]; ++t)
            (site[(size_t)t].start < c.half || !c.eo ? ev : od).push_back(site[(size_t)t]);
        for (size_t k = 0; k < ev.size() || k < od.size(); ++k) {
            if (k < ev.size()) mixed.push_back(ev[k]);
            if (k < od.size()) mixed.push_back(od[k]);
        }
    }
    e->n_half_tiles = (int64_t)half.size();
    e->n_site_tiles = (int64_t)site.size();
    // Sub-sweep layouts of the SU(3) FP64 sweep: work items of 128, 64 or 32
    // sites, in chain order or with the largest chains first; a CTA takes
    // 128 / item sites items, padded with chain = -1 items.
    std::vector<std::vector<Tile>> lay(ym::kSweepLayouts);
    {
        std::vector<int64_t> chain_order((size_t)e->n_chains), by_volume;
        for (int64_t ch = 0; ch < e->n_chains; ++ch) chain_order[(size_t)ch] = ch;
        by_volume = chain_order;
        std::stable_sort(by_volume.begin(), by_volume.end(), [&](int64_t a, int64_t b) {
            return e->chains[(size_t)a].volume > e->chains[(size_t)b].volume;
        });
        for (int li = 0; li < ym::kSweepLayouts; ++li) {
            const int log2 = 7 - li / 2;
            const int64_t g = int64_t(1) << log2, per = ym::kSweepThreads / g;
            for (int64_t ch : (li % 2) ? by_volume : chain_order)
                for (int64_t s0 = 0; s0 < e->chains[(size_t)ch].half; s0 += g)
                    lay[(size_t)li].push_back(Tile{(int32_t)ch, 0, s0});
            while ((int64_t)lay[(size_t)li].size() % per) lay[(size_t)li].push_back(Tile{-1, 0, 0});
            e->layouts[li].ctas = (int64_t)lay[(size_t)li].size() / per;
            e->layouts[li].log2_item = log2;
            e->layouts[li].by_volume = li % 2;
        }
    }
    // each chain's CTA range in the 128-site layouts (one chain per CTA, a
    // chain's CTAs consecutive)
    std::vector<std::vector<int32_t>> chain_ctas(ym::kSweepLayouts);
    for (int li = 0; li < ym::kSweepLayouts; ++li) {
        if (e->layouts[li].log2_item != 7) continue;
        std::vector<int32_t> &r = chain_ctas[(size_t)li];
        r.assign(2 * (size_t)e->n_chains, 0);
        std::vector<bool> seen((size_t)e->n_chains, false);
        for (size_t b = 0; b < lay[(size_t)li].size(); ++b) {
            const int32_t ch = lay[(size_t)li][b].chain;
            if (ch < 0) continue;
            if (!seen[(size_t)ch]) r[2 * (size_t)ch] = (int32_t)b;
            seen[(size_t)ch] = true;
            r[2 * (size_t)ch + 1] = (int32_t)b + 1;
        }
    }

    cudaError_t err = cudaSetDevice(e->device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = dalloc(&e->d_chains, e->chains.size());
    if (err == cudaSuccess) err = dalloc(&e->d_half_tiles, half.size());
    if (err == cudaSuccess) err = dalloc(&e->d_site_tiles, site.size());
    if (err == cudaSuccess) err = dalloc(&e->d_mixed_tiles, mixed.size());
    if (err == cudaSuccess) err = dalloc(&e->d_site_tile_first, first.size());
    if (err == cudaSuccess) err = dalloc(&e->d_links, (size_t)e->total_elems);
    if (err == cudaSuccess) err = dalloc(&e->d_staging, (size_t)e->max_chain_links * 18);
    if (err == cudaSuccess) err = dalloc(&e->d_partial, site.size());
    if (err == cudaSuccess) err = dalloc(&e->d_partial2, site.size());
    if (err == cudaSuccess) err = dalloc(&e->d_result, (size_t)e->n_chains);
    if (err == cudaSuccess) err = dalloc(&e->d_result2, (size_t)e->n_chains);
    if (err == cudaSuccess) err = dalloc(&e->d_accepts, (size_t)e->n_chains);
    if (err == cudaSuccess) err = dalloc(&e->d_sweep, 1);
    if (err == cudaSuccess) err = dalloc(&e->d_rng, (size_t)e->n_chains);
    if (err == cudaSuccess) err = dalloc(&e->d_ref_counts, 2 * (size_t)e->n_chains);
    if (err == cudaSuccess) err = dalloc(&e->d_error, 1);
    if (err == cudaSuccess) err = cudaMemset(e->d_error, 0, sizeof(unsigned));
    // plaquette shares of a measured sweep: three arrays of the 128-site
    // layouts' CTA count (binary64 SU(3))
    if (err == cudaSuccess && e->group == YM_GROUP_SU3 && e->precision == YM_PREC_F64)
        err = dalloc(&e->d_tr_partial, 3 * (size_t)e->layouts[0].ctas);
    if (err == cudaSuccess)
        err = cudaMemcpy(e->d_chains, e->chains.data(), e->chains.size() * sizeof(ChainInfo), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !half.empty())
        err = cudaMemcpy(e->d_half_tiles, half.data(), half.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    for (int li = 0; li < ym::kSweepLayouts && err == cudaSuccess; ++li) {
        if (!chain_ctas[(size_t)li].empty()) {
            err = dalloc(&e->layouts[li].d_chain_ctas, chain_ctas[(size_t)li].size());
            if (err == cudaSuccess)
                err = cudaMemcpy(e->layouts[li].d_chain_ctas, chain_ctas[(size_t)li].data(),
                                 chain_ctas[(size_t)li].size() * sizeof(int32_t), cudaMemcpyHostToDevice);
            if (err != cudaSuccess) break;
        }
        err = dalloc(&e->layouts[li].d_items, lay[(size_t)li].size());
        if (err == cudaSuccess && !lay[(size_t)li].empty())
            err = cudaMemcpy(e->layouts[li].d_items, lay[(size_t)li].data(), lay[(size_t)li].size() * sizeof(Tile),
                             cudaMemcpyHostToDevice);
    }
    if (err == cudaSuccess && !site.empty())
        err = cudaMemcpy(e->d_site_tiles, site.data(), site.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    if (err == cudaSuccess && !mixed.empty())
        err = cudaMemcpy(e->d_mixed_tiles, mixed.data(), mixed.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    if (err == cudaSuccess)
        err = cudaMemcpy(e->d_site_tile_first, first.data(), first.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(e->d_accepts, 0, (size_t)e->n_chains * sizeof(unsigned long long));
    if (err == cudaSuccess) err = cudaMemset(e->d_sweep, 0, sizeof(uint64_t));
    if (err == cudaSuccess) err = identity(e);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) {
        free_all(e);
        delete e;
        if (err == cudaErrorMemoryAllocation) return YM_ERR_ALLOCATION_FAILED;
        return cuda_status(err);
    }
    *out = e;
    return YM_OK;
}

int32_t ym_ensemble_destroy(ym_ensemble *e) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_all(e);
    delete e;
    return YM_OK;
}

int32_t ym_ensemble_info(const ym_ensemble *e, int64_t *n_chains, int64_t *total_links,
                         int32_t *group, int32_t *precision) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (n_chains) *n_chains = e->n_chains;
    if (total_links) *total_links = e->total_links;
    if (group) *group = e->group;
    if (precision) *precision = e->precision;
    return YM_OK;
}

int32_t ym_ensemble_set_identity(ym_ensemble *e) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(identity(e));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_hot_start(ym_ensemble *e) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(f32(e) ? ym::launch_f32_hot_start(e) : ym::launch_su3_hot_start(e));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_upload(ym_ensemble *e, int64_t chain, const double *host) {
    if (!e || !host) return YM_ERR_NULL_ARGUMENT;
    if (chain < 0 || chain >= e->n_chains) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    const size_t bytes = (size_t)e->chain_links[chain] * reals_per_link(e) * sizeof(double);
    YM_CUDA(cudaMemcpyAsync(e->d_staging, host, bytes, cudaMemcpyHostToDevice, e->stream));
    YM_CUDA(from_aos(e, chain));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_download(ym_ensemble *e, int64_t chain, double *host) {
    if (!e || !host) return YM_ERR_NULL_ARGUMENT;
    if (chain < 0 || chain >= e->n_chains) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    const size_t bytes = (size_t)e->chain_links[chain] * reals_per_link(e) * sizeof(double);
    YM_CUDA(to_aos(e, chain));
    YM_CUDA(cudaMemcpyAsync(host, e->d_staging, bytes, cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_set_sweep_index(ym_ensemble *e, uint64_t sweep) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaMemcpyAsync(e->d_sweep, &sweep, sizeof sweep, cudaMemcpyHostToDevice, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_get_sweep_index(ym_ensemble *e, uint64_t *sweep) {
    if (!e || !sweep) return YM_ERR_NULL_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaMemcpyAsync(sweep, e->d_sweep, sizeof *sweep, cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_set_chain(ym_ensemble *e, int64_t chain, double beta, uint64_t chain_seed) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (chain < 0 || chain >= e->n_chains) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    e->chains[chain].beta = beta;
    e->chains[chain].seed = chain_seed;
    YM_CUDA(cudaMemcpyAsync(e->d_chains + chain, &e->chains[chain], sizeof(ChainInfo),
                            cudaMemcpyHostToDevice, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_synchronize(ym_ensemble *e) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_ensemble_stream(ym_ensemble *e, void **stream) {
    if (!e || !stream) return YM_ERR_NULL_ARGUMENT;
    *stream = (void *)e->stream;
    return YM_OK;
}

int32_t ym_su3_metropolis_sweeps(ym_ensemble *e, double angle, int32_t generator_mode,
                                 int64_t n_sweeps) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    // metropolis_sweep validates beta before the angle (su3_ensemble.rs:348-351)
    int32_t st = validate_su3_betas(e);
    if (st) return st;
    st = validate_angle_for(e, angle);
    if (st) return st;
    if (generator_mode != YM_GEN_ORDERED && generator_mode != YM_GEN_UNIFORM) return YM_ERR_INVALID_ARGUMENT;
    if (n_sweeps < 0) return YM_ERR_INVALID_ARGUMENT;
    st = require_checkerboard(e);
    if (st) return st;
    st = set_device(e);
    if (st) return st;
    auto one_sweep = [&]() -> cudaError_t {
        for (int parity = 0; parity < 2; ++parity)
            for (int mu = 0; mu < 4; ++mu) {
                cudaError_t err = timed(e, YM_KERNEL_SU3_METROPOLIS, [&] {
                    return f32(e) ? ym::launch_f32_metropolis(e, parity, mu, angle, generator_mode)
                                  : ym::launch_su3_metropolis(e, parity, mu, angle, generator_mode);
                });
                if (err != cudaSuccess) return err;
            }
        // Two-row storage is reunitarised after every sweep: updates that
        // touch the rebuilt third row feed its norm error back into the
        // stored rows, so without it the deviation grows geometrically.
        if (f32(e)) {
            cudaError_t err = timed(e, YM_KERNEL_AUX, [&] { return ym::launch_f32_reunitarize(e); });
            if (err != cudaSuccess) return err;
        }
        return ym::launch_advance_sweep(e);
    };
    int64_t done = 0;
    // Several chains in binary64: the first call long enough times
    // kTuneSweeps sweeps on each sub-sweep layout (item size, chain order)
    // and keeps the fastest.  Every layout gives the same bits, so the probe
    // sweeps are ordinary sweeps of the chains.
    if (!f32(e) && e->n_chains > 1 && !e->layout_tuned && !e->profiling &&
        n_sweeps >= kLayoutTuneMin) {
        float best = 0.f;
        int32_t pick = 0;
        YM_CUDA(one_sweep());   // first launches (module loading) outside the probes
        done += 1;
        for (int li = 0; li < ym::kSweepLayouts; ++li) {
            e->sweep_layout = li;
            float t = 0.f;
            YM_CUDA(time_on_stream(e, [&] {
                cudaError_t err = cudaSuccess;
                for (int64_t k = 0; k < kTuneSweeps && err == cudaSuccess; ++k) err = one_sweep();
                return err;
            }, &t));
            if (li == 0 || t < best) {
                best = t;
                pick = li;
            }
            done += kTuneSweeps;
        }
        set_layout(e, pick);
        e->layout_tuned = true;
    }
    // Small chains: the first call long enough times kTuneSweeps sweeps on
    // each path and keeps the faster; the rest go to the chosen path.
    if (resident_candidate(e) && n_sweeps - done >= 2 * kTuneSweeps) {
        if (e->resident_choice < 0) {
            float t_tiled = 0.f, t_res = 0.f;
            YM_CUDA(time_on_stream(e, [&] {
                cudaError_t err = cudaSuccess;
                for (int64_t k = 0; k < kTuneSweeps && err == cudaSuccess; ++k) err = one_sweep();
                return err;
            }, &t_tiled));
            YM_CUDA(time_on_stream(e, [&] {
                return ym::launch_su3_resident(e, angle, generator_mode, 1, kTuneSweeps, nullptr);
            }, &t_res));
            e->resident_choice = t_res < t_tiled ? 1 : 0;
            done += 2 * kTuneSweeps;
        }
    }
    if (resident_candidate(e)) {
        if (e->resident_choice == 1 && done < n_sweeps) {
            YM_CUDA(ym::launch_su3_resident(e, angle, generator_mode, 1, n_sweeps - done, nullptr));
            done = n_sweeps;
        }
    }
    // Batches of kGraphSweeps sweeps replay one captured graph (9 launches
    // per sweep become one graph launch per batch).  Timed runs launch
    // directly so each kernel keeps its event pair.
    if (!e->profiling && n_sweeps - done >= kGraphSweeps) {
        if (!e->sweep_graph || e->sweep_graph_angle != angle || e->sweep_graph_mode != generator_mode) {
            if (e->sweep_graph) cudaGraphExecDestroy(e->sweep_graph);
            e->sweep_graph = nullptr;
            cudaGraph_t g = nullptr;
            YM_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t err = cudaSuccess;
            for (int k = 0; k < kGraphSweeps && err == cudaSuccess; ++k) err = one_sweep();
            cudaError_t end = cudaStreamEndCapture(e->stream, &g);
            if (err == cudaSuccess) err = end;
            if (err == cudaSuccess) err = cudaGraphInstantiate(&e->sweep_graph, g, 0);
            if (g) cudaGraphDestroy(g);
            YM_CUDA(err);
            e->sweep_graph_angle = angle;
            e->sweep_graph_mode = generator_mode;
        }
        for (; done + kGraphSweeps <= n_sweeps; done += kGraphSweeps)
            YM_CUDA(cudaGraphLaunch(e->sweep_graph, e->stream));
    }
    for (; done < n_sweeps; ++done) YM_CUDA(one_sweep());
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)n_sweeps * 32u * (uint64_t)e->chains[ch].volume;
    return YM_OK;
}

}  // extern "C"

// The per-measurement plaquette series buffer (rows x chains) and its device
// row counter.  The captured measurement graph stores into d_series by
// address, so growing the buffer also drops that graph: a graph replayed
// after the reallocation would write into the freed buffer.
static void drop_run_graph(ym_ensemble *e) {
    if (e->run_graph) cudaGraphExecDestroy(e->run_graph);
    e->run_graph = nullptr;
}

// The run_chain cadence's plaquette after a sweep.  For binary64 handles
// with ordered hits, one chain per sub-sweep CTA and chains too large for
// the chain-resident kernel, the sweep's last three sub-sweeps (parity 1,
// directions 1, 2, 3) also sum, per CTA, (1/3) Re Tr(U' A_p) of their links,
// A_p the staple terms of the lower directions: all those links are final
// then, and each plaquette of plane (nu, mu) holds exactly one odd-site
// mu-link, so the three sums are the six planes' plaquettes and no
// plaquette kernel runs.  The average plaquette agrees with
// ym_average_plaquette's to rounding (different summation order).
static bool fused_plaquette(const ym_ensemble *e, int mode) {
    return e->group == YM_GROUP_SU3 && !f32(e) && mode == YM_GEN_ORDERED && e->d_tr_partial &&
           e->layouts[e->sweep_layout].d_chain_ctas && !ym::resident_fits(e);
}

// One sweep of the cadence (measure: sub-sweeps (1, mu), mu = 1..3, also
// write their plaquette shares to d_tr_partial, one array of CTAs each).
static cudaError_t cadence_sweep(ym_ensemble *e, double angle, int mode, bool measure) {
    const int64_t ctas = e->layouts[e->sweep_layout].ctas;
    for (int parity = 0; parity < 2; ++parity)
        for (int mu = 0; mu < 4; ++mu) {
            cudaError_t err;
            if (f32(e)) err = ym::launch_f32_metropolis(e, parity, mu, angle, mode);
            else if (measure && parity == 1 && mu >= 1)
                err = ym::launch_su3_metropolis_measure(e, mu, angle, e->d_tr_partial + (mu - 1) * ctas);
            else err = ym::launch_su3_metropolis(e, parity, mu, angle, mode);
            if (err != cudaSuccess) return err;
        }
    cudaError_t err = f32(e) ? ym::launch_f32_reunitarize(e) : cudaSuccess;
    return err == cudaSuccess ? ym::launch_advance_sweep(e) : err;
}

// The average plaquette of every chain into d_result after cadence_sweep.
static cudaError_t cadence_plaquette(ym_ensemble *e, bool fused) {
    if (f32(e)) {
        cudaError_t err = ym::launch_f32_plaquette_partials(e);
        return err == cudaSuccess ? ym::launch_chain_reduce(e, e->d_partial, e->d_result, 0, 6.0) : err;
    }
    return fused ? ym::launch_su3_plaquette_from_sweep(e, e->d_tr_partial) : ym::launch_su3_plaquette(e);
}

static cudaError_t ensure_series(ym_ensemble *e, int64_t n_measurements) {
    if (e->series_capacity < n_measurements) {
        if (e->measure_graph) cudaGraphExecDestroy(e->measure_graph);
        e->measure_graph = nullptr;
        if (e->su2_graph) cudaGraphExecDestroy(e->su2_graph);
        e->su2_graph = nullptr;
        drop_run_graph(e);
        if (e->d_series) ym::dev_free(e->d_series);
        e->d_series = nullptr;
        e->series_capacity = 0;
        cudaError_t err = dalloc(&e->d_series, (size_t)(n_measurements * e->n_chains));
        if (err != cudaSuccess) return err;
        e->series_capacity = n_measurements;
    }
    if (!e->d_series_row) return dalloc(&e->d_series_row, 1);
    return cudaSuccess;
}

extern "C" {

int32_t ym_su3_measured_sweeps(ym_ensemble *e, double angle, int32_t generator_mode,
                               int64_t n_measurements, int64_t sweeps_per_measurement,
                               double *series) {
    if (!e || (!series && n_measurements > 0)) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    int32_t st = validate_su3_betas(e);
    if (st) return st;
    st = validate_angle_for(e, angle);
    if (st) return st;
    if (generator_mode != YM_GEN_ORDERED && generator_mode != YM_GEN_UNIFORM) return YM_ERR_INVALID_ARGUMENT;
    if (n_measurements < 0 || sweeps_per_measurement < 0) return YM_ERR_INVALID_ARGUMENT;
    st = require_checkerboard(e);
    if (st) return st;
    st = set_device(e);
    if (st) return st;
    if (n_measurements == 0) return YM_OK;
    YM_CUDA(ensure_series(e, n_measurements));
    YM_CUDA(cudaMemsetAsync(e->d_series_row, 0, sizeof(uint64_t), e->stream));
    const bool fused = sweeps_per_measurement > 0 && fused_plaquette(e, generator_mode);
    auto step = [&]() -> cudaError_t {
        for (int64_t k = 0; k < sweeps_per_measurement; ++k) {
            cudaError_t err = cadence_sweep(e, angle, generator_mode, fused && k == sweeps_per_measurement - 1);
            if (err != cudaSuccess) return err;
        }
        cudaError_t err = cadence_plaquette(e, fused);
        if (err == cudaSuccess) err = ym::launch_store_series(e, e->d_series, e->d_series_row);
        return err;
    };
    if (!e->measure_graph || e->measure_graph_angle != angle || e->measure_graph_mode != generator_mode ||
        e->measure_graph_stride != sweeps_per_measurement) {
        if (e->measure_graph) cudaGraphExecDestroy(e->measure_graph);
        e->measure_graph = nullptr;
        cudaGraph_t g = nullptr;
        YM_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t err = step();
        cudaError_t end = cudaStreamEndCapture(e->stream, &g);
        if (err == cudaSuccess) err = end;
        if (err == cudaSuccess) err = cudaGraphInstantiate(&e->measure_graph, g, 0);
        if (g) cudaGraphDestroy(g);
        YM_CUDA(err);
        e->measure_graph_angle = angle;
        e->measure_graph_mode = generator_mode;
        e->measure_graph_stride = sweeps_per_measurement;
    }
    int64_t m = 0;
    if (resident_candidate(e)) {
        // Rows written by the resident kernel go to row m of the series; the
        // tiled graph continues from the device row counter.
        if (e->resident_choice < 0 && n_measurements >= 2 && n_measurements * sweeps_per_measurement >= 2 * kTuneSweeps) {
            float t_tiled = 0.f, t_res = 0.f;
            YM_CUDA(time_on_stream(e, [&] { return cudaGraphLaunch(e->measure_graph, e->stream); }, &t_tiled));
            YM_CUDA(time_on_stream(e, [&] {
                return ym::launch_su3_resident(e, angle, generator_mode, 1, sweeps_per_measurement,
                                               e->d_series + 1 * e->n_chains);
            }, &t_res));
            e->resident_choice = t_res < t_tiled ? 1 : 0;
            m = 2;
        }
        if (e->resident_choice == 1 && m < n_measurements) {
            YM_CUDA(ym::launch_su3_resident(e, angle, generator_mode, n_measurements - m, sweeps_per_measurement,
                                            e->d_series + m * e->n_chains));
            m = n_measurements;
        }
        if (m > 0 && m < n_measurements) {
            const uint64_t row = (uint64_t)m;
            YM_CUDA(cudaMemcpyAsync(e->d_series_row, &row, sizeof row, cudaMemcpyHostToDevice, e->stream));
            YM_CUDA(cudaStreamSynchronize(e->stream));
        }
    }
    for (; m < n_measurements; ++m) YM_CUDA(cudaGraphLaunch(e->measure_graph, e->stream));
    YM_CUDA(cudaMemcpyAsync(series, e->d_series, (size_t)(n_measurements * e->n_chains) * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)(n_measurements * sweeps_per_measurement) * 32u *
                            (uint64_t)e->chains[ch].volume;
    return YM_OK;
}

static cudaError_t ensure_loop_series(ym_ensemble *e, int64_t rows) {
    if (e->loop_capacity < rows) {
        drop_run_graph(e);
        if (e->d_wilson_series) ym::dev_free(e->d_wilson_series);
        if (e->d_poly_series) ym::dev_free(e->d_poly_series);
        e->d_wilson_series = nullptr;
        e->d_poly_series = nullptr;
        e->loop_capacity = 0;
        cudaError_t err = dalloc(&e->d_wilson_series, (size_t)(rows * e->n_chains * 96));
        if (err == cudaSuccess) err = dalloc(&e->d_poly_series, (size_t)(rows * e->n_chains * 2));
        if (err != cudaSuccess) return err;
        e->loop_capacity = rows;
    }
    if (!e->d_loop_row) return dalloc(&e->d_loop_row, 1);
    return cudaSuccess;
}

int32_t ym_su3_measured_run(ym_ensemble *e, ym_ensemble *view, const ym_measured_run *run,
                            double *plaquette, double *wilson, double *polyakov) {
    if (!e || !run) return YM_ERR_NULL_ARGUMENT;
    if (run->n_blocks > 0 && (!plaquette || !wilson || !polyakov)) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    int32_t st = validate_su3_betas(e);
    if (st) return st;
    if ((st = validate_angle_for(e, run->proposal_angle))) return st;
    const int32_t mode = run->generator_mode;
    if (mode != YM_GEN_ORDERED && mode != YM_GEN_UNIFORM) return YM_ERR_INVALID_ARGUMENT;
    if (run->n_blocks < 0 || run->sweeps_per_block < 1) return YM_ERR_INVALID_ARGUMENT;
    if (run->rmax == 0 || run->tmax == 0) return YM_ERR_ZERO_RECTANGLE_EXTENT;
    if (run->rmax < 0 || run->tmax < 0 || run->rmax > 4 || run->tmax > 4) return YM_ERR_INVALID_ARGUMENT;
    if (run->polyakov_direction < 0 || run->polyakov_direction >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    if ((st = require_checkerboard(e))) return st;
    // The loops read binary64 links: a two-row handle is measured through a
    // binary64 handle of the same extents that receives its converted image.
    ym_ensemble *m = e;
    if (f32(e)) {
        if (!view) return YM_ERR_NULL_ARGUMENT;
        if (view->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
        if (view->precision != YM_PREC_F64) return YM_ERR_UNSUPPORTED_PRECISION;
        if (view->n_chains != e->n_chains || view->device != e->device) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
        for (int64_t ch = 0; ch < e->n_chains; ++ch)
            for (int d = 0; d < 4; ++d)
                if (view->chains[ch].n[d] != e->chains[ch].n[d]) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
        m = view;
    } else if (view && view != e) {
        return YM_ERR_INVALID_ARGUMENT;
    }
    if ((st = set_device(e))) return st;
    if (run->n_blocks == 0) return YM_OK;
    const int64_t spb = run->sweeps_per_block, rows = run->n_blocks * spb;
    YM_CUDA(ensure_obs_scratch(m));
    if (m != e) YM_CUDA(cudaStreamSynchronize(m->stream));   // m's earlier work is done
    YM_CUDA(ensure_series(e, rows));
    YM_CUDA(ensure_loop_series(e, run->n_blocks));
    YM_CUDA(cudaMemsetAsync(e->d_series_row, 0, sizeof(uint64_t), e->stream));
    YM_CUDA(cudaMemsetAsync(e->d_loop_row, 0, sizeof(uint64_t), e->stream));
    const double angle = run->proposal_angle;
    const bool fused = fused_plaquette(e, mode);
    auto block = [&]() -> cudaError_t {
        for (int64_t k = 0; k < spb; ++k) {
            cudaError_t err = cadence_sweep(e, angle, mode, fused);
            if (err == cudaSuccess) err = cadence_plaquette(e, fused);
            if (err == cudaSuccess) err = ym::launch_store_series(e, e->d_series, e->d_series_row);
            if (err != cudaSuccess) return err;
        }
        cudaError_t err = m != e ? ym::launch_convert(e, m) : cudaSuccess;
        if (err == cudaSuccess) err = ym::launch_wilson_loops(m, run->rmax, run->tmax, m->d_obs_partial, m->d_obs_out);
        if (err == cudaSuccess)
            err = ym::launch_store_rows(e->stream, m->d_obs_out, e->n_chains * 96, e->d_wilson_series, e->d_loop_row, 0);
        if (err == cudaSuccess) err = ym::launch_polyakov(m, run->polyakov_direction, m->d_obs_partial, m->d_obs_out);
        if (err == cudaSuccess)
            err = ym::launch_store_rows(e->stream, m->d_obs_out, e->n_chains * 2, e->d_poly_series, e->d_loop_row, 1);
        return err;
    };
    if (!e->run_graph || e->run_graph_angle != angle || e->run_graph_mode != mode || e->run_graph_sweeps != spb ||
        e->run_graph_rmax != run->rmax || e->run_graph_tmax != run->tmax ||
        e->run_graph_dir != run->polyakov_direction || e->run_graph_view != (const void *)m ||
        e->run_graph_view_links != (const void *)m->d_links) {
        drop_run_graph(e);
        cudaGraph_t g = nullptr;
        // the measurement handle's launches join the capture on e's stream
        cudaStream_t saved = m->stream;
        m->stream = e->stream;
        cudaError_t err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            err = block();
            const cudaError_t end = cudaStreamEndCapture(e->stream, &g);
            if (err == cudaSuccess) err = end;
        }
        m->stream = saved;
        if (err == cudaSuccess) err = cudaGraphInstantiate(&e->run_graph, g, 0);
        if (g) cudaGraphDestroy(g);
        YM_CUDA(err);
        e->run_graph_angle = angle;
        e->run_graph_mode = mode;
        e->run_graph_sweeps = spb;
        e->run_graph_rmax = run->rmax;
        e->run_graph_tmax = run->tmax;
        e->run_graph_dir = run->polyakov_direction;
        e->run_graph_view = m;
        e->run_graph_view_links = m->d_links;
    }
    for (int64_t b = 0; b < run->n_blocks; ++b) YM_CUDA(cudaGraphLaunch(e->run_graph, e->stream));
    YM_CUDA(cudaMemcpyAsync(plaquette, e->d_series, (size_t)(rows * e->n_chains) * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaMemcpyAsync(wilson, e->d_wilson_series, (size_t)(run->n_blocks * e->n_chains * 96) * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaMemcpyAsync(polyakov, e->d_poly_series, (size_t)(run->n_blocks * e->n_chains * 2) * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)rows * 32u * (uint64_t)e->chains[ch].volume;
    for (int64_t i = 0; i < rows * e->n_chains; ++i)
        if (!std::isfinite(plaquette[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
    for (int64_t i = 0; i < run->n_blocks * e->n_chains * 96; ++i)
        if (!std::isfinite(wilson[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
    for (int64_t i = 0; i < run->n_blocks * e->n_chains * 2; ++i)
        if (!std::isfinite(polyakov[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
    return YM_OK;
}

int32_t ym_ensemble_set_sweep_layout(ym_ensemble *e, int32_t item_sites, int32_t by_volume) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (item_sites == 0) {                  // automatic: tune again on the next long call
        set_layout(e, 0);
        e->layout_tuned = false;
        return YM_OK;
    }
    const int gi = item_sites == 128 ? 0 : (item_sites == 64 ? 1 : (item_sites == 32 ? 2 : -1));
    if (gi < 0 || (by_volume != 0 && by_volume != 1)) return YM_ERR_INVALID_ARGUMENT;
    set_layout(e, gi * 2 + by_volume);
    e->layout_tuned = true;
    return YM_OK;
}

int32_t ym_ensemble_get_sweep_layout(ym_ensemble *e, int32_t *item_sites, int32_t *by_volume,
                                     int32_t *tuned) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    const ym::SweepLayout &l = e->layouts[e->sweep_layout];
    if (item_sites) *item_sites = 1 << l.log2_item;
    if (by_volume) *by_volume = l.by_volume;
    if (tuned) *tuned = e->layout_tuned ? 1 : 0;
    return YM_OK;
}

int32_t ym_ensemble_lift_angle_cap(ym_ensemble *e, int32_t lift) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (lift && (e->group != YM_GROUP_SU3 || e->precision != YM_PREC_F32_TWO_ROW))
        return YM_ERR_UNSUPPORTED_PRECISION;
    e->angle_cap_lifted = lift != 0;
    return YM_OK;
}

int32_t ym_ensemble_set_fast_sweeps(ym_ensemble *e, int32_t on) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (on != 0 && on != 1) return YM_ERR_INVALID_ARGUMENT;
    if (on && (e->group != YM_GROUP_SU3 || e->precision != YM_PREC_F64)) return YM_ERR_UNSUPPORTED_PRECISION;
    if (e->fast_sweeps == (on != 0)) return YM_OK;
    e->fast_sweeps = on != 0;
    drop_sweep_graphs(e);
    return YM_OK;
}

int32_t ym_ensemble_get_fast_sweeps(ym_ensemble *e, int32_t *on) {
    if (!e || !on) return YM_ERR_NULL_ARGUMENT;
    *on = e->fast_sweeps ? 1 : 0;
    return YM_OK;
}

int32_t ym_ensemble_set_sweep_path(ym_ensemble *e, int32_t path) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (path != YM_PATH_AUTO && path != YM_PATH_TILED && path != YM_PATH_RESIDENT) return YM_ERR_INVALID_ARGUMENT;
    if (path == YM_PATH_RESIDENT) {
        int32_t st = set_device(e);
        if (st) return st;
        if (e->group != YM_GROUP_SU3 || e->precision != YM_PREC_F64 || e->fast_sweeps || !ym::resident_fits(e))
            return YM_ERR_INVALID_ARGUMENT;
    }
    e->resident_choice = path;
    return YM_OK;
}

int32_t ym_ensemble_get_sweep_path(ym_ensemble *e, int32_t *path) {
    if (!e || !path) return YM_ERR_NULL_ARGUMENT;
    *path = e->resident_choice;
    return YM_OK;
}

int32_t ym_su3_accounting(ym_ensemble *e, uint64_t *proposals, uint64_t *accepts) {
    if (!e || !proposals || !accepts) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaMemcpyAsync(accepts, e->d_accepts, (size_t)e->n_chains * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch) proposals[ch] = e->proposals[ch];
    return YM_OK;
}

int32_t ym_reset_accounting(ym_ensemble *e) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaMemsetAsync(e->d_accepts, 0, (size_t)e->n_chains * sizeof(unsigned long long), e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (auto &p : e->proposals) p = 0;
    return YM_OK;
}

int32_t ym_su3_reference_sweeps(ym_ensemble *e, double angle, uint64_t *rng_state,
                                int64_t n_sweeps, uint64_t *proposals, uint64_t *accepts) {
    if (!e || !rng_state) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(e); if (g__) return g__; }
    int32_t st = validate_su3_betas(e);
    if (st) return st;
    st = validate_angle(angle);
    if (st) return st;
    if (n_sweeps < 0) return YM_ERR_INVALID_ARGUMENT;
    st = set_device(e);
    if (st) return st;
    const size_t nb = (size_t)e->n_chains * sizeof(uint64_t);
    YM_CUDA(cudaMemcpyAsync(e->d_rng, rng_state, nb, cudaMemcpyHostToDevice, e->stream));
    YM_CUDA(ym::launch_su3_reference_sweeps(e, angle, n_sweeps));
    YM_CUDA(cudaMemcpyAsync(rng_state, e->d_rng, nb, cudaMemcpyDeviceToHost, e->stream));
    std::vector<unsigned long long> counts(2 * (size_t)e->n_chains);
    YM_CUDA(cudaMemcpyAsync(counts.data(), e->d_ref_counts, 2 * nb, cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        if (proposals) proposals[ch] = counts[ch];
        if (accepts) accepts[ch] = counts[e->n_chains + ch];
    }
    return YM_OK;
}

int32_t ym_su3_reference_average_plaquette(ym_ensemble *e, double *per_chain) {
    if (!e || !per_chain) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(e); if (g__) return g__; }
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ym::launch_su3_reference_plaquette(e));
    YM_CUDA(cudaMemcpyAsync(per_chain, e->d_result, (size_t)e->n_chains * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        if (!std::isfinite(per_chain[ch])) return YM_ERR_NON_FINITE_STATISTIC;
    return YM_OK;
}

int32_t ym_average_plaquette(ym_ensemble *e, double *per_chain) {
    if (!e || !per_chain) return YM_ERR_NULL_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(timed(e, YM_KERNEL_PLAQUETTE, [&] {
        if (f32(e)) {
            cudaError_t err = ym::launch_f32_plaquette_partials(e);
            return err == cudaSuccess ? ym::launch_chain_reduce(e, e->d_partial, e->d_result, 0, 6.0) : err;
        }
        if (e->group == YM_GROUP_SU3) return ym::launch_su3_plaquette(e);
        cudaError_t err = ym::launch_su2_plaquette_partials(e);
        return err == cudaSuccess ? ym::launch_chain_reduce(e, e->d_partial, e->d_result, 0, 6.0) : err;
    }));
    YM_CUDA(cudaMemcpyAsync(per_chain, e->d_result, (size_t)e->n_chains * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        if (!std::isfinite(per_chain[ch])) return YM_ERR_NON_FINITE_STATISTIC;
    return YM_OK;
}

int32_t ym_su3_max_residuals(ym_ensemble *e, double *unitarity, double *determinant) {
    if (!e || !unitarity || !determinant) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(e); if (g__) return g__; }
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ym::launch_su3_residuals(e));
    YM_CUDA(cudaMemcpyAsync(unitarity, e->d_result, (size_t)e->n_chains * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaMemcpyAsync(determinant, e->d_result2, (size_t)e->n_chains * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

// ---- observables and transformations ----

int32_t ym_su3_wilson_loops(ym_ensemble *e, int32_t rmax, int32_t tmax, double *out) {
    if (!e || !out) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(e); if (g__) return g__; }
    if (rmax == 0 || tmax == 0) return YM_ERR_ZERO_RECTANGLE_EXTENT;   // path_holonomy.rs:233-235
    if (rmax < 0 || tmax < 0 || rmax > 4 || tmax > 4) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ensure_obs_scratch(e));
    YM_CUDA(timed(e, YM_KERNEL_AUX, [&] { return ym::launch_wilson_loops(e, rmax, tmax, e->d_obs_partial, e->d_obs_out); }));
    YM_CUDA(cudaMemcpyAsync(out, e->d_obs_out, (size_t)e->n_chains * 96 * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_su3_polyakov_loops(ym_ensemble *e, int32_t direction, double *out) {
    if (!e || !out) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(e); if (g__) return g__; }
    if (direction < 0 || direction >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ensure_obs_scratch(e));
    YM_CUDA(timed(e, YM_KERNEL_AUX, [&] { return ym::launch_polyakov(e, direction, e->d_obs_partial, e->d_obs_out); }));
    YM_CUDA(cudaMemcpyAsync(out, e->d_obs_out, (size_t)e->n_chains * 2 * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_su2_wilson_loops(ym_ensemble *e, int32_t rmax, int32_t tmax, double *out) {
    if (!e || !out) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    if (e->precision != YM_PREC_F64) return YM_ERR_UNSUPPORTED_PRECISION;
    if (rmax == 0 || tmax == 0) return YM_ERR_ZERO_RECTANGLE_EXTENT;   // lib.rs:452-454
    if (rmax < 0 || tmax < 0 || rmax > 4 || tmax > 4) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ensure_obs_scratch(e));
    YM_CUDA(timed(e, YM_KERNEL_AUX, [&] {
        return ym::launch_su2_wilson_loops(e, rmax, tmax, e->d_obs_partial, e->d_obs_out);
    }));
    YM_CUDA(cudaMemcpyAsync(out, e->d_obs_out, (size_t)e->n_chains * 96 * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t i = 0; i < e->n_chains * 96; ++i)
        if (!std::isfinite(out[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
    return YM_OK;
}

int32_t ym_su2_polyakov_loops(ym_ensemble *e, int32_t direction, double *out) {
    if (!e || !out) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    if (direction < 0 || direction >= 4) return YM_ERR_DIRECTION_OUT_OF_RANGE;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ensure_obs_scratch(e));
    YM_CUDA(timed(e, YM_KERNEL_AUX, [&] { return ym::launch_su2_polyakov(e, direction, e->d_obs_partial, e->d_obs_out); }));
    std::vector<double> both((size_t)e->n_chains * 2);
    YM_CUDA(cudaMemcpyAsync(both.data(), e->d_obs_out, both.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch) {
        out[ch] = both[(size_t)ch * 2];
        if (!std::isfinite(out[ch])) return YM_ERR_NON_FINITE_OBSERVABLE;
    }
    return YM_OK;
}

int32_t ym_su3_scalar_operator_basis(ym_ensemble *e, double *plaquette, double *rectangle) {
    if (!e || !plaquette || !rectangle) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(e); if (g__) return g__; }
    int32_t st = require_cubic_spatial(e, 3);
    if (st) return st;
    st = set_device(e);
    if (st) return st;
    YM_CUDA(ensure_obs_scratch(e));
    YM_CUDA(timed(e, YM_KERNEL_OPERATORS, [&] {
        return ym::launch_operator_basis(e, e->d_site_vals, e->d_slice_chain, e->d_slice_t,
                                         e->n_slices, e->d_slice_plaq, e->d_slice_rect);
    }));
    YM_CUDA(cudaMemcpyAsync(plaquette, e->d_slice_plaq, (size_t)e->n_slices * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaMemcpyAsync(rectangle, e->d_slice_rect, (size_t)e->n_slices * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t i = 0; i < e->n_slices; ++i)
        if (!std::isfinite(plaquette[i]) || !std::isfinite(rectangle[i])) return YM_ERR_NON_FINITE_OBSERVABLE;
    return YM_OK;
}

int32_t ym_ensemble_copy(ym_ensemble *src, ym_ensemble *dst) {
    if (!src || !dst) return YM_ERR_NULL_ARGUMENT;
    if (!same_geometry(src, dst)) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    int32_t st = set_device(dst);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(src->stream));
    YM_CUDA(cudaMemcpyAsync(dst->d_links, src->d_links, (size_t)src->total_elems * sizeof(double2),
                            cudaMemcpyDeviceToDevice, dst->stream));
    YM_CUDA(cudaStreamSynchronize(dst->stream));
    return YM_OK;
}

int32_t ym_ensemble_copy_chain(ym_ensemble *src, int64_t src_chain, ym_ensemble *dst,
                               int64_t dst_chain) {
    if (!src || !dst) return YM_ERR_NULL_ARGUMENT;
    if (src_chain < 0 || src_chain >= src->n_chains || dst_chain < 0 || dst_chain >= dst->n_chains)
        return YM_ERR_INVALID_ARGUMENT;
    if (src->group != dst->group || src->precision != dst->precision || src->device != dst->device)
        return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    const ChainInfo &a = src->chains[src_chain], &b = dst->chains[dst_chain];
    for (int d = 0; d < 4; ++d)
        if (a.n[d] != b.n[d]) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    int32_t st = set_device(dst);
    if (st) return st;
    const size_t elem = f32(src) ? sizeof(float2) : sizeof(double2);
    const size_t per_link = f32(src) ? 6 : (src->group == YM_GROUP_SU3 ? 9 : 2);
    const size_t bytes = (size_t)a.volume * 4 * per_link * elem;
    YM_CUDA(cudaStreamSynchronize(src->stream));
    YM_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(dst->d_links) + (size_t)b.offset * elem,
                            reinterpret_cast<const char *>(src->d_links) + (size_t)a.offset * elem,
                            bytes, cudaMemcpyDeviceToDevice, dst->stream));
    YM_CUDA(cudaStreamSynchronize(dst->stream));
    return YM_OK;
}

int32_t ym_ensemble_copy_chains(ym_ensemble *src, int64_t src_first, ym_ensemble *dst,
                                int64_t dst_first, int64_t count) {
    if (!src || !dst) return YM_ERR_NULL_ARGUMENT;
    if (count < 0 || src_first < 0 || dst_first < 0 || src_first > src->n_chains - count ||
        dst_first > dst->n_chains - count)
        return YM_ERR_INVALID_ARGUMENT;
    if (count == 0) return YM_OK;
    if (src->group != dst->group || src->precision != dst->precision || src->device != dst->device)
        return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    for (int64_t i = 0; i < count; ++i) {
        const ChainInfo &a = src->chains[src_first + i], &b = dst->chains[dst_first + i];
        for (int d = 0; d < 4; ++d)
            if (a.n[d] != b.n[d]) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    }
    int32_t st = set_device(dst);
    if (st) return st;
    const size_t elem = f32(src) ? sizeof(float2) : sizeof(double2);
    const size_t per_link = f32(src) ? 6 : (src->group == YM_GROUP_SU3 ? 9 : 2);
    const ChainInfo &first = src->chains[src_first], &last = src->chains[src_first + count - 1];
    // chains sit back to back (offset of chain k+1 = offset of k + its size)
    const size_t bytes = (size_t)(last.offset - first.offset) * elem +
                         (size_t)last.volume * 4 * per_link * elem;
    YM_CUDA(cudaStreamSynchronize(src->stream));
    YM_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(dst->d_links) + (size_t)dst->chains[dst_first].offset * elem,
                            reinterpret_cast<const char *>(src->d_links) + (size_t)first.offset * elem,
                            bytes, cudaMemcpyDeviceToDevice, dst->stream));
    YM_CUDA(cudaStreamSynchronize(dst->stream));
    return YM_OK;
}

int32_t ym_su3_spatial_stout_smear(ym_ensemble *src, ym_ensemble *dst, double rho, int64_t levels,
                                   int32_t lift_level_cap) {
    if (!src || !dst) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(src); if (g__) return g__; }
    // validate_parameters (glueball_smearing.rs:83-108), in order
    if (!std::isfinite(rho)) return YM_ERR_NON_FINITE_RHO;
    if (rho <= 0.0 || rho > 0.25) return YM_ERR_RHO_OUT_OF_RANGE;
    if (levels < 0 || (!lift_level_cap && levels > 8)) return YM_ERR_TOO_MANY_LEVELS;
    int32_t st = require_cubic_spatial(src, 3);
    if (st) return st;
    if (!same_geometry(src, dst)) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    st = set_device(dst);
    if (st) return st;
    if (levels == 0) return src == dst ? YM_OK : ym_ensemble_copy(src, dst);
    if (!dst->d_links_tmp) YM_CUDA(dalloc(&dst->d_links_tmp, (size_t)dst->total_elems));
    YM_CUDA(cudaStreamSynchronize(src->stream));
    const double2 *in = src->d_links;
    // Levels alternate between dst's two buffers and end in its links.  In
    // place (src == dst) with an odd count the first level would write the
    // buffer it reads, so the input moves to the second buffer first.
    if (src == dst && levels % 2 == 1) {
        YM_CUDA(cudaMemcpyAsync(dst->d_links_tmp, dst->d_links, (size_t)dst->total_elems * sizeof(double2),
                                cudaMemcpyDeviceToDevice, dst->stream));
        in = dst->d_links_tmp;
    }
    for (int64_t k = 1; k <= levels; ++k) {
        double2 *out = ((levels - k) % 2 == 0) ? dst->d_links : dst->d_links_tmp;
        YM_CUDA(timed(dst, YM_KERNEL_STOUT, [&] { return ym::launch_stout_level(dst, in, out, rho, (int)(k & 1)); }));
        in = out;
    }
    return take_device_error(dst);
}

int32_t ym_su3_spatial_stride2_block(ym_ensemble *src, ym_ensemble *dst) {
    if (!src || !dst) return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(src); if (g__) return g__; }
    { const int32_t g__ = require_su3_f64(dst); if (g__) return g__; }
    // validate_geometry (glueball_blocking.rs:71-83), per chain
    for (const ChainInfo &c : src->chains) {
        if (c.n[0] != c.n[1] || c.n[1] != c.n[2]) return YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC;
        if (c.n[0] < 6) return YM_ERR_SPATIAL_EXTENT_TOO_SMALL;
        if (c.n[0] % 2 != 0) return YM_ERR_SPATIAL_EXTENT_NOT_EVEN;
    }
    if (src->n_chains != dst->n_chains || src->device != dst->device) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    for (int64_t ch = 0; ch < src->n_chains; ++ch) {
        const ChainInfo &f = src->chains[ch], &c = dst->chains[ch];
        if (c.n[0] * 2 != f.n[0] || c.n[1] * 2 != f.n[1] || c.n[2] * 2 != f.n[2] || c.n[3] != f.n[3])
            return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    }
    int32_t st = set_device(dst);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(src->stream));
    YM_CUDA(ym::launch_block(src, dst));
    return take_device_error(dst);
}

}  // extern "C"

// Validation, scratch and the captured measurement graph of `plan` (built on
// the first call with these handles and levels, kept on `sm`); on return
// sm->glueball_graph is ready to launch and need / blocked_slices give the
// output layout.
static int32_t glueball_graph(ym_ensemble *ens, ym_ensemble *sm, const ym_glueball_plan *plan, int64_t *need_out,
                              int64_t *blocked_out) {
    if (!ens || !sm || !plan) return YM_ERR_NULL_ARGUMENT;
    if (plan->n_levels < 1 || !plan->levels || plan->n_blocked < 0) return YM_ERR_INVALID_ARGUMENT;
    if (plan->n_blocked > 0 && (!plan->fine || !plan->coarse || !plan->first_chain))
        return YM_ERR_NULL_ARGUMENT;
    { const int32_t g__ = require_su3_f64(ens); if (g__) return g__; }
    if (!same_geometry(ens, sm)) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    // validate_parameters (glueball_smearing.rs:83-108) and the operator
    // basis' spatial check (glueball_operators.rs:72-91)
    if (!std::isfinite(plan->rho)) return YM_ERR_NON_FINITE_RHO;
    if (plan->rho <= 0.0 || plan->rho > 0.25) return YM_ERR_RHO_OUT_OF_RANGE;
    for (int32_t i = 0; i < plan->n_levels; ++i)
        if (plan->levels[i] < 0 || (i && plan->levels[i] < plan->levels[i - 1])) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = require_cubic_spatial(sm, 3);
    if (st) return st;
    int64_t blocked_slices = 0;
    for (int32_t g = 0; g < plan->n_blocked; ++g) {
        ym_ensemble *f = plan->fine[g], *c = plan->coarse[g];
        if (!f || !c) return YM_ERR_NULL_ARGUMENT;
        { const int32_t g__ = require_su3_f64(f); if (g__) return g__; }
        { const int32_t g__ = require_su3_f64(c); if (g__) return g__; }
        const int64_t first = plan->first_chain[g];
        if (first < 0 || first > sm->n_chains - f->n_chains || f->device != sm->device ||
            c->device != sm->device || c->n_chains != f->n_chains)
            return YM_ERR_INVALID_ARGUMENT;
        for (int64_t k = 0; k < f->n_chains; ++k) {
            const ChainInfo &a = sm->chains[first + k], &b = f->chains[k], &q = c->chains[k];
            for (int d = 0; d < 4; ++d)
                if (a.n[d] != b.n[d]) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
            // validate_geometry (glueball_blocking.rs:71-83)
            if (b.n[0] != b.n[1] || b.n[1] != b.n[2]) return YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC;
            if (b.n[0] < 6) return YM_ERR_SPATIAL_EXTENT_TOO_SMALL;
            if (b.n[0] % 2 != 0) return YM_ERR_SPATIAL_EXTENT_NOT_EVEN;
            if (q.n[0] * 2 != b.n[0] || q.n[1] * 2 != b.n[1] || q.n[2] * 2 != b.n[2] || q.n[3] != b.n[3])
                return YM_ERR_LATTICE_EXTENTS_MISMATCH;
        }
        if ((st = require_cubic_spatial(c, 3))) return st;
    }
    if ((st = set_device(sm))) return st;
    // scratch of every handle, made before any capture
    YM_CUDA(ensure_obs_scratch(sm));
    if (!sm->d_links_tmp) YM_CUDA(dalloc(&sm->d_links_tmp, (size_t)sm->total_elems));
    for (int32_t g = 0; g < plan->n_blocked; ++g) {
        YM_CUDA(ensure_obs_scratch(plan->coarse[g]));
        blocked_slices += plan->coarse[g]->n_slices;
    }
    const int64_t per_level = 2 * (sm->n_slices + blocked_slices);
    const int64_t need = per_level * plan->n_levels;
    // what a captured graph was made for: levels, handles and their buffers
    std::vector<int64_t> key;
    key.push_back(plan->n_levels);
    for (int32_t i = 0; i < plan->n_levels; ++i) key.push_back(plan->levels[i]);
    key.push_back((int64_t)(uintptr_t)ens->d_links);
    key.push_back((int64_t)(uintptr_t)sm->d_links);
    for (int32_t g = 0; g < plan->n_blocked; ++g) {
        key.push_back(plan->first_chain[g]);
        key.push_back((int64_t)(uintptr_t)plan->fine[g]->d_links);
        key.push_back((int64_t)(uintptr_t)plan->coarse[g]->d_links);
        key.push_back((int64_t)(uintptr_t)plan->coarse[g]->d_slice_plaq);
    }
    if (sm->gb_series_capacity < need) {
        if (sm->glueball_graph) cudaGraphExecDestroy(sm->glueball_graph);
        sm->glueball_graph = nullptr;
        if (sm->d_gb_series) ym::dev_free(sm->d_gb_series);
        sm->d_gb_series = nullptr;
        sm->gb_series_capacity = 0;
        YM_CUDA(dalloc(&sm->d_gb_series, (size_t)need));
        sm->gb_series_capacity = need;
    }
    // ens's own work (its sweeps) is done before the copy reads its links
    YM_CUDA(cudaStreamSynchronize(ens->stream));
    for (int32_t g = 0; g < plan->n_blocked; ++g) {
        YM_CUDA(cudaStreamSynchronize(plan->fine[g]->stream));
        YM_CUDA(cudaStreamSynchronize(plan->coarse[g]->stream));
    }
    auto measure = [&]() -> cudaError_t {
        cudaStream_t s0 = sm->stream;
        cudaError_t err = cudaMemcpyAsync(sm->d_links, ens->d_links, (size_t)sm->total_elems * sizeof(double2),
                                          cudaMemcpyDeviceToDevice, s0);
        // levels continue from the previous count, ping-ponging between the
        // handle's links and its second buffer; `cur` holds the latest level
        // (each level from the previous one, so the same links as smearing
        // from scratch), and the operators and group copies read it there
        double2 *cur = sm->d_links;
        int64_t done = 0;
        for (int32_t i = 0; i < plan->n_levels && err == cudaSuccess; ++i) {
            for (int64_t k = done; k < plan->levels[i] && err == cudaSuccess; ++k) {
                double2 *out = cur == sm->d_links ? sm->d_links_tmp : sm->d_links;
                err = ym::launch_stout_level(sm, cur, out, plan->rho, (int)((k + 1) & 1));   // the copy ends at the last tile
                cur = out;
            }
            done = plan->levels[i] > done ? plan->levels[i] : done;
            double *row = sm->d_gb_series + per_level * i;
            if (err == cudaSuccess)
                err = ym::launch_operator_basis(sm, sm->d_site_vals, sm->d_slice_chain, sm->d_slice_t,
                                                sm->n_slices, sm->d_slice_plaq, sm->d_slice_rect, cur);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(row, sm->d_slice_plaq, (size_t)sm->n_slices * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s0);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(row + sm->n_slices, sm->d_slice_rect, (size_t)sm->n_slices * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s0);
            double *brow = row + 2 * sm->n_slices;
            for (int32_t g = 0; g < plan->n_blocked && err == cudaSuccess; ++g) {
                ym_ensemble *f = plan->fine[g], *c = plan->coarse[g];
                const ChainInfo &a = sm->chains[plan->first_chain[g]];
                const ChainInfo &z = sm->chains[plan->first_chain[g] + f->n_chains - 1];
                const size_t bytes = (size_t)(z.offset - a.offset + z.volume * 36) * sizeof(double2);
                err = cudaMemcpyAsync(f->d_links, cur + a.offset, bytes, cudaMemcpyDeviceToDevice, s0);
                if (err == cudaSuccess) err = ym::launch_block(f, c);
                if (err == cudaSuccess)
                    err = ym::launch_operator_basis(c, c->d_site_vals, c->d_slice_chain, c->d_slice_t, c->n_slices,
                                                    c->d_slice_plaq, c->d_slice_rect);
                if (err == cudaSuccess)
                    err = cudaMemcpyAsync(brow, c->d_slice_plaq, (size_t)c->n_slices * sizeof(double),
                                          cudaMemcpyDeviceToDevice, s0);
                if (err == cudaSuccess)
                    err = cudaMemcpyAsync(brow + blocked_slices, c->d_slice_rect, (size_t)c->n_slices * sizeof(double),
                                          cudaMemcpyDeviceToDevice, s0);
                brow += c->n_slices;
            }
        }
        // the last level ends in the handle's own links (a copy only when
        // the total level count is odd)
        if (err == cudaSuccess && cur != sm->d_links)
            err = cudaMemcpyAsync(sm->d_links, cur, (size_t)sm->total_elems * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, s0);
        return err;
    };
    if (!sm->glueball_graph || sm->glueball_key != key || sm->glueball_rho != plan->rho) {
        if (sm->glueball_graph) cudaGraphExecDestroy(sm->glueball_graph);
        sm->glueball_graph = nullptr;
        // the blocked handles' launches join the capture on sm's stream
        std::vector<cudaStream_t> saved;
        for (int32_t g = 0; g < plan->n_blocked; ++g) {
            saved.push_back(plan->fine[g]->stream);
            saved.push_back(plan->coarse[g]->stream);
            plan->fine[g]->stream = sm->stream;
            plan->coarse[g]->stream = sm->stream;
        }
        cudaGraph_t graph = nullptr;
        cudaError_t err = cudaStreamBeginCapture(sm->stream, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            err = measure();
            const cudaError_t end = cudaStreamEndCapture(sm->stream, &graph);
            if (err == cudaSuccess) err = end;
        }
        for (int32_t g = 0; g < plan->n_blocked; ++g) {
            plan->fine[g]->stream = saved[(size_t)2 * g];
            plan->coarse[g]->stream = saved[(size_t)2 * g + 1];
        }
        if (err == cudaSuccess) err = cudaGraphInstantiate(&sm->glueball_graph, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        YM_CUDA(err);
        sm->glueball_key = key;
        sm->glueball_rho = plan->rho;
    }
    *need_out = need;
    *blocked_out = blocked_slices;
    return YM_OK;
}

extern "C" {

int32_t ym_su3_glueball_prepare(ym_ensemble *ens, ym_ensemble *sm, const ym_glueball_plan *plan) {
    int64_t need = 0, blocked_slices = 0;
    const int32_t st = glueball_graph(ens, sm, plan, &need, &blocked_slices);
    if (st) return st;
    YM_CUDA(cudaGraphUpload(sm->glueball_graph, sm->stream));
    YM_CUDA(cudaStreamSynchronize(sm->stream));
    return YM_OK;
}

int32_t ym_su3_glueball_measure(ym_ensemble *ens, ym_ensemble *sm, const ym_glueball_plan *plan,
                                double *plaquette, double *rectangle, double *blocked_plaquette,
                                double *blocked_rectangle) {
    if (!ens || !sm || !plan || !plaquette || !rectangle) return YM_ERR_NULL_ARGUMENT;
    if (plan->n_blocked > 0 && (!blocked_plaquette || !blocked_rectangle)) return YM_ERR_NULL_ARGUMENT;
    int64_t need = 0, blocked_slices = 0;
    int32_t st = glueball_graph(ens, sm, plan, &need, &blocked_slices);
    if (st) return st;
    const int64_t per_level = 2 * (sm->n_slices + blocked_slices);
    YM_CUDA(cudaGraphLaunch(sm->glueball_graph, sm->stream));
    std::vector<double> host((size_t)need);
    YM_CUDA(cudaMemcpyAsync(host.data(), sm->d_gb_series, (size_t)need * sizeof(double), cudaMemcpyDeviceToHost,
                            sm->stream));
    YM_CUDA(cudaStreamSynchronize(sm->stream));
    // gates of the kernels that ran (stout: sm's flag, blocking: each coarse flag)
    if ((st = take_device_error(sm))) return st;
    for (int32_t g = 0; g < plan->n_blocked; ++g)
        if ((st = take_device_error(plan->coarse[g]))) return st;
    for (int32_t i = 0; i < plan->n_levels; ++i) {
        const double *row = host.data() + per_level * i;
        for (int64_t k = 0; k < sm->n_slices; ++k) {
            plaquette[i * sm->n_slices + k] = row[k];
            rectangle[i * sm->n_slices + k] = row[sm->n_slices + k];
        }
        for (int64_t k = 0; k < blocked_slices; ++k) {
            blocked_plaquette[i * blocked_slices + k] = row[2 * sm->n_slices + k];
            blocked_rectangle[i * blocked_slices + k] = row[2 * sm->n_slices + blocked_slices + k];
        }
    }
    for (int64_t k = 0; k < need; ++k)
        if (!std::isfinite(host[(size_t)k])) return YM_ERR_NON_FINITE_OBSERVABLE;
    return YM_OK;
}

int32_t ym_su3_reunitarize(ym_ensemble *e) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    if (!f32(e)) return YM_ERR_UNSUPPORTED_PRECISION;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(timed(e, YM_KERNEL_AUX, [&] { return ym::launch_f32_reunitarize(e); }));
    return YM_OK;
}

int32_t ym_ensemble_convert(ym_ensemble *src, ym_ensemble *dst) {
    if (!src || !dst) return YM_ERR_NULL_ARGUMENT;
    if (src->group != YM_GROUP_SU3 || dst->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    if (src->precision == dst->precision) return ym_ensemble_copy(src, dst);
    if (src->n_chains != dst->n_chains || src->device != dst->device) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    for (int64_t ch = 0; ch < src->n_chains; ++ch)
        for (int d = 0; d < 4; ++d)
            if (src->chains[ch].n[d] != dst->chains[ch].n[d]) return YM_ERR_LATTICE_EXTENTS_MISMATCH;
    int32_t st = set_device(dst);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(src->stream));
    YM_CUDA(ym::launch_convert(src, dst));
    YM_CUDA(cudaStreamSynchronize(dst->stream));
    return YM_OK;
}

// ---- SU(2) ----

int32_t ym_su2_markov_sweeps(ym_ensemble *e, int64_t max_attempts_per_link,
                             int64_t overrelaxation_sweeps, int32_t sampler, int64_t n_sweeps) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    // heatbath_sweep checks beta, then the attempt limit (su2_ensemble.rs:321-332)
    for (const ChainInfo &c : e->chains)
        if (!std::isfinite(c.beta) || c.beta < 0.0 || c.beta > kMaxSu2Beta)
            return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (max_attempts_per_link == 0) return YM_ERR_ZERO_HEATBATH_ATTEMPT_LIMIT;
    if (max_attempts_per_link < 0 || max_attempts_per_link > (int64_t(1) << 30) ||
        overrelaxation_sweeps < 0 || n_sweeps < 0 || (sampler != YM_SU2_SAMPLER_REFERENCE &&
                                                      sampler != YM_SU2_SAMPLER_KENNEDY_PENDLETON))
        return YM_ERR_INVALID_ARGUMENT;
    int32_t st = require_checkerboard(e);
    if (st) return st;
    st = set_device(e);
    if (st) return st;
    for (int64_t sw = 0; sw < n_sweeps; ++sw) {
        for (int parity = 0; parity < 2; ++parity)
            for (int mu = 0; mu < 4; ++mu)
                YM_CUDA(timed(e, YM_KERNEL_SU2_HEATBATH, [&] {
                    return ym::launch_su2_heatbath(e, parity, mu, (int)max_attempts_per_link, sampler);
                }));
        YM_CUDA(ym::launch_advance_sweep(e));
        for (int64_t k = 0; k < overrelaxation_sweeps; ++k)
            for (int parity = 0; parity < 2; ++parity)
                for (int mu = 0; mu < 4; ++mu)
                    YM_CUDA(timed(e, YM_KERNEL_SU2_OVERRELAX, [&] {
                        return ym::launch_su2_overrelax(e, parity, mu);
                    }));
    }
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)n_sweeps * 4u * (uint64_t)e->chains[ch].volume;
    return take_device_error(e);
}

int32_t ym_su2_measured_sweeps(ym_ensemble *e, int64_t max_attempts_per_link, int64_t overrelaxation_sweeps,
                               int32_t sampler, int64_t n_measurements, int64_t sweeps_per_measurement,
                               double *series) {
    if (!e || (!series && n_measurements > 0)) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    for (const ChainInfo &c : e->chains)
        if (!std::isfinite(c.beta) || c.beta < 0.0 || c.beta > kMaxSu2Beta)
            return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
    if (max_attempts_per_link == 0) return YM_ERR_ZERO_HEATBATH_ATTEMPT_LIMIT;
    if (max_attempts_per_link < 0 || max_attempts_per_link > (int64_t(1) << 30) || overrelaxation_sweeps < 0 ||
        n_measurements < 0 || sweeps_per_measurement < 0 ||
        (sampler != YM_SU2_SAMPLER_REFERENCE && sampler != YM_SU2_SAMPLER_KENNEDY_PENDLETON))
        return YM_ERR_INVALID_ARGUMENT;
    int32_t st = require_checkerboard(e);
    if (st) return st;
    st = set_device(e);
    if (st) return st;
    if (n_measurements == 0) return YM_OK;
    YM_CUDA(ensure_series(e, n_measurements));
    YM_CUDA(cudaMemsetAsync(e->d_series_row, 0, sizeof(uint64_t), e->stream));
    // one measurement: the sweeps of ym_su2_markov_sweeps, then the average
    // plaquette of every chain into the next row of the device series
    auto step = [&]() -> cudaError_t {
        cudaError_t err = cudaSuccess;
        for (int64_t k = 0; k < sweeps_per_measurement && err == cudaSuccess; ++k) {
            for (int parity = 0; parity < 2 && err == cudaSuccess; ++parity)
                for (int mu = 0; mu < 4 && err == cudaSuccess; ++mu)
                    err = ym::launch_su2_heatbath(e, parity, mu, (int)max_attempts_per_link, sampler);
            if (err == cudaSuccess) err = ym::launch_advance_sweep(e);
            for (int64_t o = 0; o < overrelaxation_sweeps && err == cudaSuccess; ++o)
                for (int parity = 0; parity < 2 && err == cudaSuccess; ++parity)
                    for (int mu = 0; mu < 4 && err == cudaSuccess; ++mu) err = ym::launch_su2_overrelax(e, parity, mu);
        }
        if (err == cudaSuccess) err = ym::launch_su2_plaquette_partials(e);
        if (err == cudaSuccess) err = ym::launch_chain_reduce(e, e->d_partial, e->d_result, 0, 6.0);
        if (err == cudaSuccess) err = ym::launch_store_series(e, e->d_series, e->d_series_row);
        return err;
    };
    const int64_t key[4] = {max_attempts_per_link, overrelaxation_sweeps, sampler, sweeps_per_measurement};
    if (!e->su2_graph || !std::equal(key, key + 4, e->su2_graph_key)) {
        if (e->su2_graph) cudaGraphExecDestroy(e->su2_graph);
        e->su2_graph = nullptr;
        cudaGraph_t g = nullptr;
        YM_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t err = step();
        const cudaError_t end = cudaStreamEndCapture(e->stream, &g);
        if (err == cudaSuccess) err = end;
        if (err == cudaSuccess) err = cudaGraphInstantiate(&e->su2_graph, g, 0);
        if (g) cudaGraphDestroy(g);
        YM_CUDA(err);
        std::copy(key, key + 4, e->su2_graph_key);
    }
    for (int64_t m = 0; m < n_measurements; ++m) YM_CUDA(cudaGraphLaunch(e->su2_graph, e->stream));
    YM_CUDA(cudaMemcpyAsync(series, e->d_series, (size_t)(n_measurements * e->n_chains) * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)(n_measurements * sweeps_per_measurement) * 4u * (uint64_t)e->chains[ch].volume;
    st = take_device_error(e);
    if (st) return st;
    for (int64_t k = 0; k < n_measurements * e->n_chains; ++k)
        if (!std::isfinite(series[k])) return YM_ERR_NON_FINITE_STATISTIC;
    return YM_OK;
}

int32_t ym_su2_overrelaxation_sweeps(ym_ensemble *e, int64_t n_sweeps) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    if (n_sweeps < 0) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = require_checkerboard(e);
    if (st) return st;
    st = set_device(e);
    if (st) return st;
    for (int64_t k = 0; k < n_sweeps; ++k)
        for (int parity = 0; parity < 2; ++parity)
            for (int mu = 0; mu < 4; ++mu)
                YM_CUDA(timed(e, YM_KERNEL_SU2_OVERRELAX, [&] { return ym::launch_su2_overrelax(e, parity, mu); }));
    return take_device_error(e);
}

int32_t ym_su2_accounting(ym_ensemble *e, uint64_t *proposals, uint64_t *updates) {
    if (!e || !proposals || !updates) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaMemcpyAsync(proposals, e->d_accepts, (size_t)e->n_chains * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch) updates[ch] = e->proposals[ch];
    return YM_OK;
}

int32_t ym_su2_max_unit_residual(ym_ensemble *e, double *per_chain) {
    if (!e || !per_chain) return YM_ERR_NULL_ARGUMENT;
    if (e->group != YM_GROUP_SU2) return YM_ERR_WRONG_GROUP;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(ym::launch_su2_unit_residual_partials(e));
    YM_CUDA(ym::launch_chain_reduce(e, e->d_partial, e->d_result, 1, 1.0));
    YM_CUDA(cudaMemcpyAsync(per_chain, e->d_result, (size_t)e->n_chains * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    YM_CUDA(cudaStreamSynchronize(e->stream));
    return YM_OK;
}

int32_t ym_profile_enable(ym_ensemble *e, int32_t on) {
    if (!e) return YM_ERR_NULL_ARGUMENT;
    e->profiling = on != 0;
    for (size_t &u : e->events_used) u = 0;
    return YM_OK;
}

int32_t ym_profile_read(ym_ensemble *e, int32_t kernel, double *total_ms, int64_t *launches) {
    if (!e || !total_ms || !launches) return YM_ERR_NULL_ARGUMENT;
    if (kernel < 0 || kernel >= YM_KERNEL_COUNT) return YM_ERR_INVALID_ARGUMENT;
    int32_t st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(e->stream));
    double ms = 0.0;
    for (size_t i = 0; i < e->events_used[kernel]; ++i) {
        float t = 0.0f;
        YM_CUDA(cudaEventElapsedTime(&t, e->events[kernel][i].start, e->events[kernel][i].stop));
        ms += t;
    }
    *total_ms = ms;
    *launches = (int64_t)e->events_used[kernel];
    e->events_used[kernel] = 0;
    return YM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ learned proposal
namespace {

void free_model(ym_proposal_model *m) {
    void *ptrs[] = {m->d_params, m->d_adam_m, m->d_adam_v, m->d_image, m->d_error, m->d_feat,
                    m->d_mrec, m->d_b3, m->d_y, m->d_partial, m->d_groups, m->d_grad, m->d_objective};
    for (void *p : ptrs)
        if (p) ym::dev_free(p);
    if (m->stream) cudaStreamDestroy(m->stream);
}

int32_t model_device(const ym_proposal_model *m) { return cuda_status(cudaSetDevice(m->device)); }

cudaError_t ensure_rows(ym_proposal_model *m, int64_t rows) {
    rows = (rows + 127) / 128 * 128;
    if (rows <= m->row_capacity) return cudaSuccess;
    float **bufs[] = {&m->d_feat, &m->d_mrec, &m->d_b3, &m->d_y};
    for (float **b : bufs)
        if (*b) {
            ym::dev_free(*b);
            *b = nullptr;
        }
    m->row_capacity = 0;
    cudaError_t err = dalloc(&m->d_feat, (size_t)rows * 16);
    if (err == cudaSuccess) err = dalloc(&m->d_mrec, (size_t)rows * 18);
    if (err == cudaSuccess) err = dalloc(&m->d_b3, (size_t)rows);
    if (err == cudaSuccess) err = dalloc(&m->d_y, (size_t)rows * 16);
    if (err == cudaSuccess) m->row_capacity = rows;
    return err;
}

cudaError_t ensure_partials(ym_proposal_model *m, int64_t tiles) {
    if (tiles <= m->partial_capacity) return cudaSuccess;
    if (m->d_partial) ym::dev_free(m->d_partial);
    if (m->d_groups) ym::dev_free(m->d_groups);
    m->d_partial = nullptr;
    m->d_groups = nullptr;
    m->partial_capacity = 0;
    cudaError_t err = dalloc(&m->d_partial, (size_t)(tiles * ym::kLpPartialStride));
    if (err == cudaSuccess)
        err = dalloc(&m->d_groups, (size_t)(ym::lp_reduce_groups(tiles) * ym::kLpPartialStride));
    if (err == cudaSuccess) m->partial_capacity = tiles;
    return err;
}

cudaError_t ensure_objectives(ym_proposal_model *m, int64_t n) {
    if (n <= m->objective_capacity) return cudaSuccess;
    if (m->d_objective) ym::dev_free(m->d_objective);
    m->d_objective = nullptr;
    m->objective_capacity = 0;
    cudaError_t err = dalloc(&m->d_objective, (size_t)n);
    if (err == cudaSuccess) m->objective_capacity = n;
    return err;
}

// Outputs 9..15 are padding: their weights and biases stay zero.
void zero_padding(float *p) {
    for (int i = YM_LP_OFF_W3 + 9 * 64; i < YM_LP_OFF_B3; ++i) p[i] = 0.0f;
    for (int i = YM_LP_OFF_B3 + 9; i < YM_LP_PARAMS; ++i) p[i] = 0.0f;
}

int32_t upload_params(ym_proposal_model *m, const float *host) {
    std::vector<float> p(host, host + YM_LP_PARAMS);
    zero_padding(p.data());
    for (float v : p)
        if (!std::isfinite(v)) return YM_ERR_INVALID_ARGUMENT;
    YM_CUDA(cudaMemcpyAsync(m->d_params, p.data(), sizeof(float) * YM_LP_PARAMS, cudaMemcpyHostToDevice,
                            m->stream));
    YM_CUDA(cudaMemsetAsync(m->d_adam_m, 0, sizeof(float) * YM_LP_PARAMS, m->stream));
    YM_CUDA(cudaMemsetAsync(m->d_adam_v, 0, sizeof(float) * YM_LP_PARAMS, m->stream));
    YM_CUDA(cudaMemsetAsync(m->d_image, 0, 12288, m->stream));
    YM_CUDA(ym::launch_lp_image(m, m->stream));
    YM_CUDA(cudaStreamSynchronize(m->stream));
    m->adam_step = 0;
    return YM_OK;
}

// Reads and clears the model's device error bits after `st` drains.
int32_t take_model_error(ym_proposal_model *m, cudaStream_t st) {
    unsigned bits = 0;
    YM_CUDA(cudaMemcpyAsync(&bits, m->d_error, sizeof bits, cudaMemcpyDeviceToHost, st));
    YM_CUDA(cudaStreamSynchronize(st));
    if (!bits) return YM_OK;
    YM_CUDA(cudaMemsetAsync(m->d_error, 0, sizeof(unsigned), st));
    YM_CUDA(cudaStreamSynchronize(st));
    return YM_ERR_DEVICE_WAIT_TIMEOUT;
}

int32_t require_learned(const ym_ensemble *e, const ym_proposal_model *m) {
    if (e->group != YM_GROUP_SU3) return YM_ERR_WRONG_GROUP;
    if (e->precision != YM_PREC_F32_TWO_ROW) return YM_ERR_UNSUPPORTED_PRECISION;
    int32_t st = validate_su3_betas(e);
    if (st) return st;
    st = require_checkerboard(e);
    if (st) return st;
    if (m && m->device != e->device) return YM_ERR_INVALID_ARGUMENT;
    return YM_OK;
}

cudaError_t plain_uniform_sweep(ym_ensemble *e, double angle) {
    for (int parity = 0; parity < 2; ++parity)
        for (int mu = 0; mu < 4; ++mu) {
            cudaError_t err = ym::launch_f32_metropolis(e, parity, mu, angle, YM_GEN_UNIFORM);
            if (err != cudaSuccess) return err;
        }
    cudaError_t err = ym::launch_f32_reunitarize(e);
    return err == cudaSuccess ? ym::launch_advance_sweep(e) : err;
}

cudaError_t learned_sweep(ym_ensemble *e, ym_proposal_model *m) {
    for (int parity = 0; parity < 2; ++parity)
        for (int mu = 0; mu < 4; ++mu) {
            cudaError_t err = timed(e, YM_KERNEL_LEARNED, [&] { return ym::launch_lp_sweep(e, m, parity, mu); });
            if (err != cudaSuccess) return err;
        }
    cudaError_t err = timed(e, YM_KERNEL_AUX, [&] { return ym::launch_f32_reunitarize(e); });
    return err == cudaSuccess ? ym::launch_advance_sweep(e) : err;
}

int64_t half_sites(const ym_ensemble *e) {
    int64_t n = 0;
    for (const ChainInfo &c : e->chains) n += c.half;
    return n;
}

}  // namespace

extern "C" {

int32_t ym_device_wait_selftest(int32_t device, int64_t limit_ns) {
    if (limit_ns < 1000 || limit_ns > 1000000000) return YM_ERR_INVALID_ARGUMENT;
    YM_CUDA(cudaSetDevice(device));
    unsigned *d_err = nullptr;
    YM_CUDA(dalloc(&d_err, 1));
    unsigned bits = 0;
    cudaError_t err = cudaMemset(d_err, 0, sizeof(unsigned));
    if (err == cudaSuccess) err = ym::launch_lp_wait_selftest((uint64_t)limit_ns, d_err, nullptr);
    if (err == cudaSuccess) err = cudaMemcpy(&bits, d_err, sizeof bits, cudaMemcpyDeviceToHost);
    ym::dev_free(d_err);
    YM_CUDA(err);
    return bits ? YM_ERR_DEVICE_WAIT_TIMEOUT : YM_OK;
}

int32_t ym_model_create(int32_t device, uint64_t seed, double initial_scale, ym_proposal_model **out) {
    if (!out) return YM_ERR_NULL_ARGUMENT;
    *out = nullptr;
    if (!std::isfinite(initial_scale) || initial_scale <= YM_LP_SCALE_MIN || initial_scale >= YM_LP_SCALE_MAX)
        return YM_ERR_INVALID_ARGUMENT;
    ym_proposal_model *m = new (std::nothrow) ym_proposal_model();
    if (!m) return YM_ERR_CUDA;
    m->device = device;
    auto fail = [&](int32_t st) {
        free_model(m);
        delete m;
        return st;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(cuda_status(cudaSetDevice(device)));
    cudaError_t err = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = dalloc(&m->d_params, YM_LP_PARAMS);
    if (err == cudaSuccess) err = dalloc(&m->d_adam_m, YM_LP_PARAMS);
    if (err == cudaSuccess) err = dalloc(&m->d_adam_v, YM_LP_PARAMS);
    if (err == cudaSuccess) err = dalloc(&m->d_grad, YM_LP_PARAMS);
    if (err == cudaSuccess) err = dalloc(&m->d_image, 12288);
    if (err == cudaSuccess) err = dalloc(&m->d_error, 1);
    if (err == cudaSuccess) err = cudaMemset(m->d_error, 0, sizeof(unsigned));
    if (err != cudaSuccess) return fail(cuda_status(err));
    // He-uniform draw from a SplitMix64 stream of the seed; the last layer
    // scaled by 1/8; zero biases except the scale output.
    std::vector<float> p(YM_LP_PARAMS, 0.0f);
    uint64_t n = 0;
    auto uniform = [&](double bound) {
        const double u = (double)(ym_splitmix64_at(seed, n++) >> 11) * (1.0 / 9007199254740992.0);
        return (float)((2.0 * u - 1.0) * bound);
    };
    for (int i = 0; i < 64 * 16; ++i) p[YM_LP_OFF_W1 + i] = uniform(std::sqrt(6.0 / 16.0));
    for (int i = 0; i < 64 * 64; ++i) p[YM_LP_OFF_W2 + i] = uniform(std::sqrt(6.0 / 64.0));
    for (int i = 0; i < 9 * 64; ++i) p[YM_LP_OFF_W3 + i] = uniform(std::sqrt(6.0 / 64.0) / 8.0);
    const double q = (initial_scale - YM_LP_SCALE_MIN) / (YM_LP_SCALE_MAX - YM_LP_SCALE_MIN);
    p[YM_LP_OFF_B3 + 8] = (float)std::log(q / (1.0 - q));
    const int32_t st = upload_params(m, p.data());
    if (st) return fail(st);
    *out = m;
    return YM_OK;
}

int32_t ym_model_destroy(ym_proposal_model *m) {
    if (!m) return YM_ERR_NULL_ARGUMENT;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    free_model(m);
    delete m;
    return YM_OK;
}

int32_t ym_model_get_params(ym_proposal_model *m, float *params) {
    if (!m || !params) return YM_ERR_NULL_ARGUMENT;
    int32_t st = model_device(m);
    if (st) return st;
    YM_CUDA(cudaMemcpyAsync(params, m->d_params, sizeof(float) * YM_LP_PARAMS, cudaMemcpyDeviceToHost,
                            m->stream));
    YM_CUDA(cudaStreamSynchronize(m->stream));
    return YM_OK;
}

int32_t ym_model_set_params(ym_proposal_model *m, const float *params) {
    if (!m || !params) return YM_ERR_NULL_ARGUMENT;
    int32_t st = model_device(m);
    if (st) return st;
    return upload_params(m, params);
}

int32_t ym_model_forward(ym_proposal_model *m, const float *features, int64_t n, float *outputs) {
    if (!m || ((!features || !outputs) && n > 0)) return YM_ERR_NULL_ARGUMENT;
    if (n < 0) return YM_ERR_INVALID_ARGUMENT;
    if (n == 0) return YM_OK;
    int32_t st = model_device(m);
    if (st) return st;
    YM_CUDA(ensure_rows(m, n));
    YM_CUDA(cudaMemcpyAsync(m->d_feat, features, sizeof(float) * 16 * (size_t)n, cudaMemcpyHostToDevice,
                            m->stream));
    YM_CUDA(ym::launch_lp_forward(m, m->d_feat, n, m->d_y, m->stream));
    YM_CUDA(cudaMemcpyAsync(outputs, m->d_y, sizeof(float) * 16 * (size_t)n, cudaMemcpyDeviceToHost,
                            m->stream));
    return take_model_error(m, m->stream);
}

int32_t ym_model_gradient(ym_proposal_model *m, const float *features, const float *mrec,
                          const double *beta, int64_t n, double *objective, float *grad) {
    if (!m || !features || !mrec || !beta || !objective || !grad) return YM_ERR_NULL_ARGUMENT;
    if (n <= 0) return YM_ERR_INVALID_ARGUMENT;
    std::vector<float> b3((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        if (!std::isfinite(beta[i]) || beta[i] < 0.0 || beta[i] > kMaxSu3Beta)
            return YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE;
        b3[(size_t)i] = (float)(beta[i] / 3.0);
    }
    int32_t st = model_device(m);
    if (st) return st;
    const int64_t tiles = (n + 127) / 128;
    YM_CUDA(ensure_rows(m, n));
    YM_CUDA(ensure_partials(m, tiles));
    YM_CUDA(ensure_objectives(m, 1));
    YM_CUDA(cudaMemcpyAsync(m->d_feat, features, sizeof(float) * 16 * (size_t)n, cudaMemcpyHostToDevice, m->stream));
    YM_CUDA(cudaMemcpyAsync(m->d_mrec, mrec, sizeof(float) * 18 * (size_t)n, cudaMemcpyHostToDevice, m->stream));
    YM_CUDA(cudaMemcpyAsync(m->d_b3, b3.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, m->stream));
    YM_CUDA(ym::launch_lp_grad(m, m->d_feat, m->d_mrec, m->d_b3, n, m->stream));
    YM_CUDA(ym::launch_lp_adam(m, tiles, n, 0.0f, 0, m->d_grad, m->d_objective, m->stream));
    YM_CUDA(cudaMemcpyAsync(grad, m->d_grad, sizeof(float) * YM_LP_PARAMS, cudaMemcpyDeviceToHost, m->stream));
    YM_CUDA(cudaMemcpyAsync(objective, m->d_objective, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    return take_model_error(m, m->stream);
}

int32_t ym_learned_records(ym_ensemble *e, int32_t parity, int32_t mu, float *features, float *mrec,
                           double *beta, int64_t *n_out) {
    if (!e || !n_out) return YM_ERR_NULL_ARGUMENT;
    int32_t st = require_learned(e, nullptr);
    if (st) return st;
    if (parity < 0 || parity > 1 || mu < 0 || mu > 3) return YM_ERR_INVALID_ARGUMENT;
    *n_out = half_sites(e);
    if (!features || !mrec || !beta) return YM_OK;
    st = set_device(e);
    if (st) return st;
    const int64_t rows = e->n_half_tiles * 128;
    float *d_f = nullptr, *d_m = nullptr, *d_b = nullptr;
    cudaError_t err = dalloc(&d_f, (size_t)rows * 16);
    if (err == cudaSuccess) err = dalloc(&d_m, (size_t)rows * 18);
    if (err == cudaSuccess) err = dalloc(&d_b, (size_t)rows);
    std::vector<float> hf, hm;
    if (err == cudaSuccess) err = ym::launch_lp_records(e, parity, mu, d_f, d_m, d_b);
    if (err == cudaSuccess) {
        hf.resize((size_t)rows * 16);
        hm.resize((size_t)rows * 18);
        err = cudaMemcpyAsync(hf.data(), d_f, hf.size() * sizeof(float), cudaMemcpyDeviceToHost, e->stream);
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(hm.data(), d_m, hm.size() * sizeof(float), cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    ym::dev_free(d_f);
    ym::dev_free(d_m);
    ym::dev_free(d_b);
    YM_CUDA(err);
    // tiles are laid out chain by chain, 128 sites of the parity each
    int64_t tile0 = 0, out = 0;
    for (const ChainInfo &c : e->chains) {
        for (int64_t t = 0; t < c.half; ++t, ++out) {
            const int64_t row = tile0 * 128 + t;
            std::memcpy(features + out * 16, hf.data() + row * 16, 16 * sizeof(float));
            std::memcpy(mrec + out * 18, hm.data() + row * 18, 18 * sizeof(float));
            beta[out] = c.beta;
        }
        tile0 += (c.half + 127) / 128;
    }
    return YM_OK;
}

int32_t ym_model_train(ym_proposal_model *m, ym_ensemble *e, int64_t n_steps, int64_t sweeps_per_step,
                       double plain_angle, double lr, double *objective_history) {
    if (!m || !e) return YM_ERR_NULL_ARGUMENT;
    int32_t st = require_learned(e, m);
    if (st) return st;
    st = validate_angle(plain_angle);
    if (st) return st;
    if (n_steps < 0 || sweeps_per_step < 0 || !std::isfinite(lr) || lr <= 0.0) return YM_ERR_INVALID_ARGUMENT;
    if (n_steps == 0) return YM_OK;
    st = set_device(e);
    if (st) return st;
    const int64_t rows = e->n_half_tiles * 128;
    YM_CUDA(ensure_rows(m, rows));
    YM_CUDA(ensure_partials(m, e->n_half_tiles));
    YM_CUDA(ensure_objectives(m, n_steps));
    YM_CUDA(cudaStreamSynchronize(m->stream));   // model-stream work before ensemble-stream work
    const int64_t n_valid = half_sites(e);
    for (int64_t step = 0; step < n_steps; ++step) {
        for (int64_t k = 0; k < sweeps_per_step; ++k) YM_CUDA(plain_uniform_sweep(e, plain_angle));
        const int sub = (int)(step % 8);
        YM_CUDA(ym::launch_lp_records(e, sub / 4, sub % 4, m->d_feat, m->d_mrec, m->d_b3));
        YM_CUDA(ym::launch_lp_grad(m, m->d_feat, m->d_mrec, m->d_b3, rows, e->stream));
        YM_CUDA(ym::launch_lp_adam(m, e->n_half_tiles, n_valid, (float)lr, 1, nullptr,
                                   m->d_objective + step, e->stream));
    }
    if (objective_history)
        YM_CUDA(cudaMemcpyAsync(objective_history, m->d_objective, sizeof(double) * (size_t)n_steps,
                                cudaMemcpyDeviceToHost, e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)(n_steps * sweeps_per_step) * 32u * (uint64_t)e->chains[ch].volume;
    return take_model_error(m, e->stream);
}

int32_t ym_su3_learned_sweeps(ym_ensemble *e, ym_proposal_model *m, int64_t n_sweeps) {
    if (!e || !m) return YM_ERR_NULL_ARGUMENT;
    int32_t st = require_learned(e, m);
    if (st) return st;
    if (n_sweeps < 0) return YM_ERR_INVALID_ARGUMENT;
    st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(m->stream));
    for (int64_t k = 0; k < n_sweeps; ++k) YM_CUDA(learned_sweep(e, m));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)n_sweeps * 32u * (uint64_t)e->chains[ch].volume;
    return take_model_error(m, e->stream);
}

int32_t ym_su3_learned_measured_sweeps(ym_ensemble *e, ym_proposal_model *m, int64_t n_measurements,
                                       int64_t sweeps_per_measurement, double *series) {
    if (!e || !m || (!series && n_measurements > 0)) return YM_ERR_NULL_ARGUMENT;
    int32_t st = require_learned(e, m);
    if (st) return st;
    if (n_measurements < 0 || sweeps_per_measurement < 0) return YM_ERR_INVALID_ARGUMENT;
    if (n_measurements == 0) return YM_OK;
    st = set_device(e);
    if (st) return st;
    YM_CUDA(cudaStreamSynchronize(m->stream));
    YM_CUDA(ensure_series(e, n_measurements));
    YM_CUDA(cudaMemsetAsync(e->d_series_row, 0, sizeof(uint64_t), e->stream));
    for (int64_t meas = 0; meas < n_measurements; ++meas) {
        for (int64_t k = 0; k < sweeps_per_measurement; ++k) YM_CUDA(learned_sweep(e, m));
        YM_CUDA(ym::launch_f32_plaquette_partials(e));
        YM_CUDA(ym::launch_chain_reduce(e, e->d_partial, e->d_result, 0, 6.0));
        YM_CUDA(ym::launch_store_series(e, e->d_series, e->d_series_row));
    }
    YM_CUDA(cudaMemcpyAsync(series, e->d_series, (size_t)(n_measurements * e->n_chains) * sizeof(double),
                            cudaMemcpyDeviceToHost, e->stream));
    for (int64_t ch = 0; ch < e->n_chains; ++ch)
        e->proposals[ch] += (uint64_t)(n_measurements * sweeps_per_measurement) * 32u *
                            (uint64_t)e->chains[ch].volume;
    return take_model_error(m, e->stream);
}

}  // extern "C"
