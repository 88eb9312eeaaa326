// ym_internal.hpp -- host-side state of an ensemble handle and the launcher
// interface between the C ABI (capi.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/ymgpu.h"
#include "ym_device.cuh"

namespace ym {

constexpr int kSweepThreads = 128;   // threads per tile of a sub-sweep
constexpr int kSiteThreads = 128;    // threads per tile of a measurement
constexpr int64_t kLpPartialStride = 6304;  // floats per tile of learned-proposal gradient partials
// Groups of 64 tiles in the first stage of the gradient reduction.
inline int64_t lp_reduce_groups(int64_t tiles) { return (tiles + 63) / 64; }

// Maps a CUDA error onto a status (YM_OK or YM_ERR_CUDA) and records a
// failure as the calling thread's ym_last_cuda_error (capi.cu).
int32_t record_cuda_status(cudaError_t err);

// One work layout of the SU(3) FP64 sub-sweep: a table of work items of
// 2^log2_item sites (a 128-thread CTA takes 128 >> log2_item of them, so
// items of different chains can share a CTA), padded with chain = -1 items
// to whole CTAs.
struct SweepLayout {
    Tile *d_items = nullptr;
    int64_t ctas = 0;
    int32_t log2_item = 7;
    int32_t by_volume = 0;     // items of the largest chains first
    // 128-site items (one chain per CTA): [2 * chain] first CTA, [2 * chain + 1]
    // one past the last CTA of each chain; null for the other item sizes
    int32_t *d_chain_ctas = nullptr;
};
constexpr int kSweepLayouts = 6;   // item sizes 128, 64, 32 x (chain order, by volume)

}  // namespace ym

struct ym_ensemble {
    int32_t group = 3;
    int32_t precision = YM_PREC_F64;
    int32_t device = 0;
    int64_t n_chains = 0;
    std::vector<ym::ChainInfo> chains;     // host copy
    std::vector<int64_t> chain_links;      // links per chain
    int64_t total_links = 0;
    int64_t max_chain_links = 0;
    int64_t total_elems = 0;               // double2 elements of link storage

    ym::ChainInfo *d_chains = nullptr;
    ym::Tile *d_half_tiles = nullptr;      // work items = checkerboard half
    int64_t n_half_tiles = 0;
    ym::Tile *d_site_tiles = nullptr;      // work items = all sites
    ym::Tile *d_mixed_tiles = nullptr;     // the same tiles, each chain's even and odd halves
                                           // interleaved (order-free per-site kernels whose
                                           // neighbours are the other parity: stout smearing)
    int64_t n_site_tiles = 0;
    int32_t *d_site_tile_first = nullptr;  // first site tile of each chain (+ end)

    double2 *d_links = nullptr;
    double *d_staging = nullptr;           // AoS image of one chain
    double *d_partial = nullptr;           // one double per site tile
    double *d_partial2 = nullptr;          // second partial per site tile
    double *d_result = nullptr;            // n_chains results
    double *d_result2 = nullptr;
    unsigned long long *d_accepts = nullptr;   // SU(3) accepts / SU(2) heat-bath attempts
    unsigned *d_error = nullptr;               // device error bits (bounded loops that gave up)
    double *d_tr_partial = nullptr;            // 3 x CTAs: plaquette shares of a measured sweep
    uint64_t *d_sweep = nullptr;           // next sweep index
    uint64_t *d_rng = nullptr;             // reference-replay stream states
    unsigned long long *d_ref_counts = nullptr;  // reference replay: proposals, accepts
    std::vector<uint64_t> proposals;       // host-counted proposals per chain

    cudaStream_t stream = nullptr;

    // Measurement scratch, allocated on first use.
    double *d_obs_partial = nullptr;       // n_site_tiles * 96
    double *d_obs_out = nullptr;           // n_chains * 96
    double2 *d_site_vals = nullptr;        // one double2 per site
    int32_t *d_slice_chain = nullptr;      // (chain, t) of every time slice
    int32_t *d_slice_t = nullptr;
    double *d_slice_plaq = nullptr;
    double *d_slice_rect = nullptr;
    int64_t n_slices = 0;
    double2 *d_links_tmp = nullptr;        // second link buffer (smearing levels)

    // Lattice queries (lattice_ops.cu), allocated on first use.
    unsigned *d_query_error = nullptr;     // error bits of the running query
    double *d_query = nullptr;             // 64 doubles: single-site results and arguments
    int32_t *d_steps = nullptr;            // a path's steps
    int64_t steps_capacity = 0;
    double *d_terms = nullptr;             // per-plaquette action terms of one chain
    int64_t terms_capacity = 0;

    // Captured batch of sweeps, replayed by ym_su3_metropolis_sweeps (the
    // sweep index lives in device memory, so every replay advances it).
    cudaGraphExec_t sweep_graph = nullptr;
    double sweep_graph_angle = 0.0;
    int32_t sweep_graph_mode = -1;
    // Captured "sweeps then plaquette into the series" step.
    cudaGraphExec_t measure_graph = nullptr;
    double measure_graph_angle = 0.0;
    int32_t measure_graph_mode = -1;
    int64_t measure_graph_stride = -1;
    // SU(2) measurement graph (ym_su2_measured_sweeps) and what it was made
    // for: attempt limit, overrelaxation sweeps, sampler, sweeps per row.
    cudaGraphExec_t su2_graph = nullptr;
    int64_t su2_graph_key[4] = {-1, -1, -1, -1};
    // Small-chain path choice: -1 not yet measured, 0 tiled launches, 1 the
    // chain-resident kernel (picked by timing both on the first sweeps).
    int32_t resident_choice = -1;
    // Sub-sweep layouts of the SU(3) FP64 sweep and the one in use (picked
    // by timing each on the first long sweep call of a handle with several
    // chains, or set by the caller).
    ym::SweepLayout layouts[ym::kSweepLayouts];
    int32_t sweep_layout = 0;
    bool layout_tuned = false;
    // Half widths above the reference's 1.0 admitted (two-row handles only).
    bool angle_cap_lifted = false;
    // SU(3) FP64 sweeps in the fast form (fused multiply-adds, Horner
    // rotations; su3_metropolis_fast.cu) instead of the reference's bits.
    bool fast_sweeps = false;
    // Captured block of the loop-measurement cadence (ym_su3_measured_run):
    // sweeps with a plaquette each, then Wilson and Polyakov loops.
    cudaGraphExec_t run_graph = nullptr;
    double run_graph_angle = 0.0;
    int32_t run_graph_mode = -1;
    int64_t run_graph_sweeps = -1;
    int32_t run_graph_rmax = 0, run_graph_tmax = 0, run_graph_dir = -1;
    const void *run_graph_view = nullptr;      // measurement handle and its buffers
    const void *run_graph_view_links = nullptr;
    double *d_wilson_series = nullptr;     // [block][chain][96]
    double *d_poly_series = nullptr;       // [block][chain][2]
    int64_t loop_capacity = 0;             // rows
    uint64_t *d_loop_row = nullptr;
    // Captured glueball measurement (ym_su3_glueball_measure), kept on the
    // smeared handle: the graph, what it was captured for, and its outputs
    // [level][slice] for this handle and for the blocked handles.
    cudaGraphExec_t glueball_graph = nullptr;
    std::vector<int64_t> glueball_key;
    double glueball_rho = 0.0;
    double *d_gb_series = nullptr;
    int64_t gb_series_capacity = 0;        // doubles
    double *d_series = nullptr;            // [measurement][chain]
    int64_t series_capacity = 0;           // rows
    uint64_t *d_series_row = nullptr;

    // Optional per-kernel timing: event pairs bracket each launch.
    bool profiling = false;
    struct EventPair { cudaEvent_t start, stop; };
    std::vector<EventPair> events[8];
    size_t events_used[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// A learned-proposal model on one device (include/ym_learned.h).
struct ym_proposal_model {
    int32_t device = 0;
    float *d_params = nullptr;             // YM_LP_PARAMS fp32 master parameters
    float *d_adam_m = nullptr;
    float *d_adam_v = nullptr;
    int64_t adam_step = 0;
    uint8_t *d_image = nullptr;            // BF16 weights in the shared-memory tile layout
    unsigned *d_error = nullptr;           // bit 0: a tensor-core wait gave up
    // Training and inspection buffers, grown on demand.
    float *d_feat = nullptr;               // [rows][16]
    float *d_mrec = nullptr;               // [rows][18]
    float *d_b3 = nullptr;                 // [rows], negative marks a padding row
    float *d_y = nullptr;                  // [rows][16]
    int64_t row_capacity = 0;
    float *d_partial = nullptr;            // [tiles][kLpPartialStride]
    int64_t partial_capacity = 0;
    double *d_groups = nullptr;            // [ceil(tiles / 64)][kLpPartialStride]
    float *d_grad = nullptr;               // YM_LP_PARAMS
    double *d_objective = nullptr;         // per training step
    int64_t objective_capacity = 0;
    cudaStream_t stream = nullptr;
};

namespace ym {

// learned.cu
cudaError_t launch_lp_records(ym_ensemble *e, int parity, int mu, float *feat, float *m, float *b3);
cudaError_t launch_lp_image(ym_proposal_model *m, cudaStream_t st);
cudaError_t launch_lp_forward(ym_proposal_model *m, const float *feat, int64_t n, float *y,
                              cudaStream_t st);
cudaError_t launch_lp_grad(ym_proposal_model *m, const float *feat, const float *mrec,
                           const float *b3, int64_t n, cudaStream_t st);
cudaError_t launch_lp_adam(ym_proposal_model *m, int64_t n_tiles, int64_t n_valid, float lr,
                           int update, float *grad_out, double *objective_out, cudaStream_t st);
cudaError_t launch_lp_sweep(ym_ensemble *e, ym_proposal_model *m, int parity, int mu);
cudaError_t launch_lp_wait_selftest(uint64_t limit_ns, unsigned *err, cudaStream_t st);

// Launchers implemented in su3_f64.cu (return a cudaError_t).
cudaError_t launch_su3_identity(ym_ensemble *e);
cudaError_t launch_su3_from_aos(ym_ensemble *e, int64_t chain);
cudaError_t launch_su3_to_aos(ym_ensemble *e, int64_t chain);
// Device memory of the library (capi.cu): from the current device's
// stream-ordered pool, ready for every stream on return; dev_free gives a
// block back to the pool of the device that holds it.
cudaError_t dev_alloc(void **ptr, size_t bytes);
void dev_free(void *ptr);
cudaError_t launch_su3_metropolis(ym_ensemble *e, int parity, int mu, double angle, int uniform);
// The same sub-sweep in the fast form (su3_metropolis_fast.cu);
// launch_su3_metropolis dispatches to it when e->fast_sweeps is set.
cudaError_t launch_su3_metropolis_fast(ym_ensemble *e, int parity, int mu, double angle, int uniform);
// Sub-sweep (parity 1, mu), mu = 1, 2 or 3, with ordered hits, also writing
// each CTA's share of the plaquettes in planes (nu, mu), nu < mu, to
// tr_partial[cta]; the handle's layout must hold one chain per CTA.
cudaError_t launch_su3_metropolis_measure(ym_ensemble *e, int mu, double angle, double *tr_partial);
cudaError_t launch_su3_metropolis_measure_fast(ym_ensemble *e, int mu, double angle, double *tr_partial);
// After a sweep whose last three sub-sweeps measured into tr_partial
// (three arrays of the layout's CTA count): each chain's average plaquette
// into d_result.
cudaError_t launch_su3_plaquette_from_sweep(ym_ensemble *e, const double *tr_partial);
cudaError_t launch_advance_sweep(ym_ensemble *e);
// Chain-resident sweeps (su3_metropolis.cu): every chain small enough that
// its links fit in one CTA's shared memory.  series (device, may be null)
// receives the plaquette of every chain after each group of sweeps.
bool resident_fits(const ym_ensemble *e);
cudaError_t launch_su3_resident(ym_ensemble *e, double angle, int uniform, int64_t n_meas,
                                int64_t sweeps_per_meas, double *series);
cudaError_t launch_su3_plaquette(ym_ensemble *e);
cudaError_t launch_su3_residuals(ym_ensemble *e);
cudaError_t launch_su3_reference_sweeps(ym_ensemble *e, double angle, int64_t n_sweeps);
cudaError_t launch_su3_reference_plaquette(ym_ensemble *e);
cudaError_t launch_su3_hot_start(ym_ensemble *e);
cudaError_t launch_chain_reduce(ym_ensemble *e, const double *partial, double *out, int mode,
                                double per_site);
cudaError_t launch_store_series(ym_ensemble *e, double *series, uint64_t *counter);
// Row *counter of dst (rows of n doubles) = src; advance bumps the counter.
cudaError_t launch_store_rows(cudaStream_t st, const double *src, int64_t n, double *dst,
                              uint64_t *counter, int advance);

// observables.cu / smear.cu
cudaError_t launch_wilson_loops(ym_ensemble *e, int rmax, int tmax, double *d_partial, double *d_out);
cudaError_t launch_polyakov(ym_ensemble *e, int dir, double *d_partial, double *d_out);
// The operator basis of e's links, or of `links` (a buffer in e's layout)
// when given.
cudaError_t launch_operator_basis(ym_ensemble *e, double2 *d_site_vals, const int32_t *d_slice_chain,
                                  const int32_t *d_slice_t, int64_t n_slices, double *d_plaq,
                                  double *d_rect, const double2 *links = nullptr);
// One stout level in -> out.  Consecutive levels pass reverse = 0, 1, 0, ...
// so each walks its tiles opposite to the last and starts on the links the
// previous level wrote last (in L2); per-site work, so no bit changes.
cudaError_t launch_stout_level(ym_ensemble *e, const double2 *in, double2 *out, double rho, int reverse);
cudaError_t launch_block(ym_ensemble *fine, ym_ensemble *coarse);
// Per-chain means of tile partials [tile][width] (loops: / volume; dir >= 0:
// / number of lines along dir), fixed order.
cudaError_t launch_tile_mean(ym_ensemble *e, const double *d_partial, int width, int dir, double *d_out);

// lattice_ops.cu (SU(2) lattice averages of the reference's loops)
cudaError_t launch_su2_wilson_loops(ym_ensemble *e, int rmax, int tmax, double *d_partial, double *d_out);
cudaError_t launch_su2_polyakov(ym_ensemble *e, int dir, double *d_partial, double *d_out);

// su3_f32.cu (two-row binary32 storage)
cudaError_t launch_f32_metropolis(ym_ensemble *e, int parity, int mu, double angle, int uniform);
cudaError_t launch_f32_reunitarize(ym_ensemble *e);
cudaError_t launch_f32_plaquette_partials(ym_ensemble *e);
cudaError_t launch_f32_identity(ym_ensemble *e);
cudaError_t launch_f32_hot_start(ym_ensemble *e);
cudaError_t launch_f32_from_aos(ym_ensemble *e, int64_t chain);
cudaError_t launch_f32_to_aos(ym_ensemble *e, int64_t chain);
cudaError_t launch_convert(ym_ensemble *src, ym_ensemble *dst);
// One link of a two-row handle as binary64 (9 double2, third row rebuilt) /
// from binary64 (first two rows stored in binary32).
cudaError_t launch_f32_get_link(ym_ensemble *e, int64_t chain, int64_t s, int mu, double2 *out);
cudaError_t launch_f32_set_link(ym_ensemble *e, int64_t chain, int64_t s, int mu, const double2 *in);

// su2.cu
cudaError_t launch_su2_heatbath(ym_ensemble *e, int parity, int mu, int max_attempts, int kp);
cudaError_t launch_su2_overrelax(ym_ensemble *e, int parity, int mu);
cudaError_t launch_su2_plaquette_partials(ym_ensemble *e);
cudaError_t launch_su2_unit_residual_partials(ym_ensemble *e);
cudaError_t launch_su2_identity(ym_ensemble *e);
cudaError_t launch_su2_from_aos(ym_ensemble *e, int64_t chain);
cudaError_t launch_su2_to_aos(ym_ensemble *e, int64_t chain);

}  // namespace ym
