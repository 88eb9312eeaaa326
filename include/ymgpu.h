/* ymgpu.h -- C ABI of libymgpu, the B200 (sm_100a) lattice gauge engine.
 *
 * Drop-in boundary for the data-parallel path of QSOLKCB/YANG-MILLS: link
 * sweeps, gauge observables and glueball measurements.  The reference exposes
 * that path as module-level Rust functions over owned host lattices
 * (`Su3Lattice4`, `Lattice4`) and a `&mut SplitMix64`; this ABI keeps the
 * same operations, argument meanings and fail-closed error behaviour, with
 * lattices held on the device:
 *
 *   - an opaque `ym_ensemble` owns the device links of one or more chains
 *     (one chain = one reference lattice; many chains of uneven extents can
 *     share one handle and are updated by the same kernel launches);
 *   - host lattices cross the boundary in the reference's own memory order
 *     (`Vec<Su3>`/`Vec<Su2>` with link index site*4+mu, lexicographic sites,
 *     x3 fastest; SU(3) = 18 doubles row-major re/im, SU(2) = 4 doubles);
 *   - every call returns an int32 `ym_status` (include/ym_status.h), results
 *     come back through caller-owned out-pointers, nothing panics;
 *   - calls on one handle are not thread-safe (the reference takes
 *     `&mut lattice`); each handle owns one CUDA stream.
 *
 * Random numbers: the reference draws from one SplitMix64 stream in
 * lexicographic link order.  A checkerboard engine cannot split that stream,
 * so every link visit owns a counter-based SplitMix64 stream keyed by
 * (chain seed, sweep index, link):  key = S(S(seed, sweep), 4*site+mu) with
 * S(k, n) = mix64(k + (n+1)*0x9E3779B97F4A7C15), the reference's own
 * generator evaluated at a given position.  The per-link update rule and its
 * arithmetic are the reference's.  ym_su3_reference_sweeps additionally
 * replays the reference's single-stream lexicographic order bit for bit.
 */
#ifndef YMGPU_H
#define YMGPU_H

#include <stddef.h>
#include <stdint.h>

#include "ym_analysis.h"
#include "ym_config.h"
#include "ym_learned.h"
#include "ym_status.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ym_ensemble ym_ensemble;

/* The cudaError_t behind the calling thread's most recent YM_ERR_CUDA. */
int32_t ym_last_cuda_error(void);

enum { YM_GROUP_SU2 = 2, YM_GROUP_SU3 = 3 };

/* Link storage precision.  F64 keeps all 18 reals of an SU(3) link;
 * F32_TWO_ROW keeps the first two rows in binary32 (12 reals) and rebuilds
 * the third as the conjugate cross product. */
enum { YM_PREC_F64 = 0, YM_PREC_F32_TWO_ROW = 1 };

/* SU(3) Metropolis generator choice.  ORDERED: the reference's eight hits per
 * link, generators 1..8 in order (su3_ensemble.rs:361).  UNIFORM: eight hits,
 * each generator drawn uniformly from bits 52..54 of the hit's angle word
 * (bits the angle grid does not use). */
enum { YM_GEN_ORDERED = 0, YM_GEN_UNIFORM = 1 };

typedef struct {
    int32_t group;                /* YM_GROUP_SU2 or YM_GROUP_SU3 */
    int32_t precision;            /* YM_PREC_* */
    int64_t n_chains;             /* >= 1 */
    const int64_t *extents;       /* n_chains x 4, every extent >= 2 */
    const double *beta;           /* n_chains couplings (may differ) */
    const uint64_t *chain_seed;   /* n_chains stream seeds */
    int32_t lift_reference_caps;  /* 0: reject lattices above the reference's
                                     link caps (2^18 SU(3), 2^20 SU(2)) */
    int32_t device;               /* CUDA device ordinal */
} ym_ensemble_desc;

/* ---- handle lifetime (Su3Lattice4::new_identity su3_lattice.rs:85,
 *      Lattice4::new_identity lib.rs:242) ---- */
int32_t ym_ensemble_create(const ym_ensemble_desc *desc, ym_ensemble **out);
int32_t ym_ensemble_destroy(ym_ensemble *ens);
int32_t ym_ensemble_info(const ym_ensemble *ens, int64_t *n_chains, int64_t *total_links,
                         int32_t *group, int32_t *precision);
/* Device memory (no reference counterpart): handles draw their device
 * buffers from the device's default stream-ordered memory pool, and what a
 * destroyed handle frees stays in that pool for the next handle (creating
 * and destroying handles then costs well under a millisecond).  Other code
 * in the process that allocates with cudaMalloc sees the pooled memory as
 * taken; this call gives the pool's unused memory on `device` back to the
 * driver, after waiting for the device to go idle. */
int32_t ym_device_release_pooled_memory(int32_t device);
/* Cold start: every link the identity (all chains). */
int32_t ym_ensemble_set_identity(ym_ensemble *ens);
/* Hot start (no reference counterpart: the reference always starts cold,
 * su3_ensemble.rs:412): every SU(3) link Haar-random, drawn from a stream
 * keyed by the chain seed and the link index. */
int32_t ym_ensemble_hot_start(ym_ensemble *ens);
/* Copy one chain's links from/to a host array in the reference layout.
 * Blocking with respect to the host buffer. */
int32_t ym_ensemble_upload(ym_ensemble *ens, int64_t chain, const double *host_links);
int32_t ym_ensemble_download(ym_ensemble *ens, int64_t chain, double *host_links);
/* Sweep counter: the index the next sweep uses in the stream key. */
int32_t ym_ensemble_set_sweep_index(ym_ensemble *ens, uint64_t sweep);
int32_t ym_ensemble_get_sweep_index(ym_ensemble *ens, uint64_t *sweep);
int32_t ym_ensemble_synchronize(ym_ensemble *ens);
/* The handle's CUDA stream (cudaStream_t), for callers that order their own
 * work after the engine's. */
int32_t ym_ensemble_stream(ym_ensemble *ens, void **stream);

/* ---- SU(3) Metropolis (su3_ensemble.rs:342-391 metropolis_sweep) ----
 * n_sweeps checkerboard sweeps of every chain: parity 0 then 1, direction
 * 0..3, eight hits per link visit, accept iff u < exp(-max(dS,0)).  Every
 * extent must be even (YM_ERR_NOT_CHECKERBOARDABLE).  proposal_angle is the
 * paired-grid half width, validated as in the reference (1e-8 <= a <= 1);
 * beta per chain must lie in [0, 12]. */
int32_t ym_su3_metropolis_sweeps(ym_ensemble *ens, double proposal_angle, int32_t generator_mode,
                                 int64_t n_sweeps);
/* The run_chain measurement cadence (su3_ensemble.rs:424-435) without a host
 * round trip per measurement: n_measurements times {sweeps_per_measurement
 * sweeps, average plaquette of every chain}, replayed from one captured CUDA
 * graph; series[m * n_chains + chain] receives measurement m.  The sweeps
 * are those of ym_su3_metropolis_sweeps bit for bit.  For binary64 handles
 * with ordered hits whose chains are too large for the chain-resident
 * kernel, the plaquette comes from the sweep itself: sub-sweeps (parity 1,
 * direction mu = 1, 2, 3) before each measurement also sum, over their
 * links, Re Tr(U'A_p) with A_p the staple terms of the directions below mu,
 * which are exactly the plaquettes of the planes (nu, mu), nu < mu.  The
 * series is then within 1e-12 relative of ym_average_plaquette (another
 * summation order); otherwise it is ym_average_plaquette's bit for bit.
 * ym_su3_measured_run measures the same way. */
int32_t ym_su3_measured_sweeps(ym_ensemble *ens, double proposal_angle, int32_t generator_mode,
                               int64_t n_measurements, int64_t sweeps_per_measurement,
                               double *series);
/* The run_chain cadence with loop observables (su3_ensemble.rs:408-480 for
 * the sweep/measure order; the loops are path_holonomy.rs:172-260 and
 * su3_lattice.rs:185-212 averaged over the lattice): n_blocks times
 *   { sweeps_per_block x (one sweep, the average plaquette of every chain),
 *     Wilson loops R x T <= rmax x tmax of every chain (ym_su3_wilson_loops),
 *     Polyakov loops along polyakov_direction (ym_su3_polyakov_loops) },
 * each block replayed from one captured CUDA graph with no host round trip.
 * A two-row binary32 handle sweeps with binary64 reunitarisation after every
 * sweep and an FP64 plaquette; its loops are measured on `view`, a binary64
 * handle of the same extents that receives the converted links every block
 * (for a binary64 handle `view` is NULL or the handle itself).
 *   plaquette [n_blocks * sweeps_per_block][n_chains]
 *   wilson    [n_blocks][n_chains][96] (layout of ym_su3_wilson_loops)
 *   polyakov  [n_blocks][n_chains][2]  (mean re, im) */
typedef struct {
    double proposal_angle;
    int32_t generator_mode;        /* YM_GEN_* */
    int32_t polyakov_direction;    /* 0..3 */
    int64_t n_blocks;              /* loop measurements */
    int64_t sweeps_per_block;      /* sweeps between loop measurements, >= 1 */
    int32_t rmax, tmax;            /* 1..4 */
} ym_measured_run;
int32_t ym_su3_measured_run(ym_ensemble *ens, ym_ensemble *view, const ym_measured_run *run,
                            double *plaquette, double *wilson, double *polyakov);
/* Sweep path of SU(3) FP64 handles (no reference counterpart).  When every
 * chain is small enough for its links to sit in one CTA's shared memory
 * (4^4 and similar), sweeps can run chain-resident: one launch does many
 * whole sweeps of every chain in shared memory.  YM_PATH_AUTO (the default)
 * times a few sweeps on each path in the first call long enough to tell
 * them apart and keeps the faster; YM_PATH_TILED and YM_PATH_RESIDENT force
 * one (RESIDENT fails with YM_ERR_INVALID_ARGUMENT when a chain does not
 * fit, the handle is not SU(3) FP64 or its fast sweeps are on).  Both paths
 * give the same bits:
 * links, accept counts and measured plaquettes. */
enum { YM_PATH_AUTO = -1, YM_PATH_TILED = 0, YM_PATH_RESIDENT = 1 };
int32_t ym_ensemble_set_sweep_path(ym_ensemble *ens, int32_t path);
/* The path in use: YM_PATH_AUTO while not yet decided. */
int32_t ym_ensemble_get_sweep_path(ym_ensemble *ens, int32_t *path);
/* Work layout of the tiled SU(3) FP64 sub-sweep (no reference counterpart):
 * the half lattice of every chain is cut into work items of item_sites
 * sites (128, 64 or 32; a 128-thread CTA takes 128 / item_sites items, so
 * the remainders of small chains share CTAs instead of leaving threads idle),
 * listed in chain order (by_volume = 0) or largest chains first (1).  On a
 * handle with several chains the first ym_su3_metropolis_sweeps call of at
 * least 50 sweeps times 4 sweeps on each of the six layouts and keeps the
 * fastest (then the chain-resident path is weighed against it as before);
 * item_sites = 0 asks for that tuning again.  Every layout gives the same
 * bits. */
int32_t ym_ensemble_set_sweep_layout(ym_ensemble *ens, int32_t item_sites, int32_t by_volume);
int32_t ym_ensemble_get_sweep_layout(ym_ensemble *ens, int32_t *item_sites, int32_t *by_volume,
                                     int32_t *tuned);

/* Fast SU(3) FP64 sweeps (no reference counterpart; off by default).  With
 * on = 1 the sweeps of a binary64 SU(3) handle run the same algorithm,
 * streams and binary64 storage with every product free to round once (fused
 * multiply-adds) and each hit's rotation entries from a Horner polynomial
 * instead of the reference's Taylor recurrence: a link moves by a few ulps
 * per update against the exact sweep (at most 9.3e-16 after one sweep and
 * 3.2e-15 after ten on a 16^4 lattice from a Haar start, every accept
 * decision unchanged), and a decision can differ only when its uniform lies
 * that close to exp(-dS).  Fast sweeps always run on the tiled path
 * (YM_PATH_RESIDENT fails with YM_ERR_INVALID_ARGUMENT while they are on);
 * other handles fail with YM_ERR_UNSUPPORTED_PRECISION. */
int32_t ym_ensemble_set_fast_sweeps(ym_ensemble *ens, int32_t on);
int32_t ym_ensemble_get_fast_sweeps(ym_ensemble *ens, int32_t *on);

/* Proposal half widths above the reference's cap of 1.0 (no reference
 * counterpart: su3_ensemble.rs:28 rejects them).  With lift != 0 the sweeps
 * of a two-row binary32 handle accept half widths up to 2.5, the range of
 * the learned proposal's scale, so that plain Metropolis can run at the
 * scale the learned proposal settles at (a matched control).  binary64
 * handles keep the reference's cap: their exact exponential assumes
 * |theta/2| < 1/2 (YM_ERR_UNSUPPORTED_PRECISION). */
int32_t ym_ensemble_lift_angle_cap(ym_ensemble *ens, int32_t lift);

/* Accumulated proposals/accepts per chain since creation or reset
 * (MetropolisAccounting su3_ensemble.rs:117-121). */
int32_t ym_su3_accounting(ym_ensemble *ens, uint64_t *proposals, uint64_t *accepts);
int32_t ym_reset_accounting(ym_ensemble *ens);

/* The reference's own sweep, replayed on the device one thread per chain:
 * lexicographic link order, one SplitMix64 stream per chain whose state is
 * read from and written back to rng_state[n_chains], twelve-plaquette action
 * difference (su3_ensemble.rs:261-391).  Slow by design; it exists so the
 * device reproduces the reference's chains exactly. */
int32_t ym_su3_reference_sweeps(ym_ensemble *ens, double proposal_angle, uint64_t *rng_state,
                                int64_t n_sweeps, uint64_t *proposals, uint64_t *accepts);
/* Lexicographic sequential plaquette sum, one thread per chain: the
 * reference's summation order (su3_ensemble.rs:228-259), bit for bit. */
int32_t ym_su3_reference_average_plaquette(ym_ensemble *ens, double *per_chain);

/* ---- SU(2) heat-bath ensemble (su2_ensemble.rs:220-552) ----
 * n_sweeps Markov sweeps of every chain, each one heat-bath sweep
 * (checkerboard parity 0 then 1, direction 0..3) followed by
 * overrelaxation_sweeps overrelaxation sweeps (markov_sweep :465-486).  The
 * heat-bath sampler is the reference's truncated-exponential inverse CDF with
 * Haar rejection (su2_ensemble.rs:220-254) or, alternatively, Kennedy-
 * Pendleton for the same density.  Each link visit draws from its own
 * counter-based stream; at most max_attempts_per_link proposals per visit,
 * after which the link keeps its value and the call returns
 * YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED (the device never waits unbounded).
 * Every extent must be even; beta per chain in [0, 8]. */
enum { YM_SU2_SAMPLER_REFERENCE = 0, YM_SU2_SAMPLER_KENNEDY_PENDLETON = 1 };
int32_t ym_su2_markov_sweeps(ym_ensemble *ens, int64_t max_attempts_per_link,
                             int64_t overrelaxation_sweeps, int32_t sampler, int64_t n_sweeps);
/* The SU(2) run_chain cadence (su2_ensemble.rs:465-486: sweeps, then the
 * average plaquette, per measurement) without a host round trip per
 * measurement: n_measurements times {sweeps_per_measurement sweeps of
 * ym_su2_markov_sweeps, average plaquette of every chain}, replayed from one
 * captured CUDA graph; series[m * n_chains + chain] receives measurement m.
 * The same links, streams and values as the separate calls; an exhausted
 * attempt limit anywhere in the run returns
 * YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED after it. */
int32_t ym_su2_measured_sweeps(ym_ensemble *ens, int64_t max_attempts_per_link, int64_t overrelaxation_sweeps,
                               int32_t sampler, int64_t n_measurements, int64_t sweeps_per_measurement,
                               double *series);
/* overrelaxation_sweep (su2_ensemble.rs:344-346), checkerboard order. */
int32_t ym_su2_overrelaxation_sweeps(ym_ensemble *ens, int64_t n_sweeps);
/* Heat-bath proposals (attempts) and updates per chain since creation or
 * reset (ChainReport::heatbath_proposals/updates su2_ensemble.rs:180-181). */
int32_t ym_su2_accounting(ym_ensemble *ens, uint64_t *proposals, uint64_t *updates);
/* Lattice4::max_link_unit_residual (lib.rs:726-740) per chain. */
int32_t ym_su2_max_unit_residual(ym_ensemble *ens, double *per_chain);

/* ---- observables ----
 * Average plaquette per chain (su3_ensemble.rs:228 / su2_ensemble.rs:348):
 * mean over sites and mu<nu of (1/N) Re Tr P, each SU(3) plaquette's two
 * matrix products as fma chains, FP64 tree reduction in a fixed order
 * (deterministic; within 1e-12 relative of the reference's sequential sum,
 * tested up to 32^4). */
int32_t ym_average_plaquette(ym_ensemble *ens, double *per_chain);
/* Average plaquette without any device allocation.  No counterpart in the
 * reference: it serves callers that cannot allocate device memory (a host
 * framework whose pool owns the device and only lends the engine buffers it
 * allocated itself, or a fixed-footprint deployment that must not call the
 * CUDA allocator after start-up).
 *   links   device pointer, 16-byte aligned, to one SU(3) lattice in the
 *           reference layout (link = site*4+mu, 18 doubles each);
 *   extents host array of 4 extents, each >= 2;
 *   out     device pointer receiving one double, the average plaquette:
 *           within 1e-12 relative of ym_average_plaquette's value (the two
 *           sum in different orders, so they need not agree bit for bit;
 *           it is not checked for finiteness);
 *   stream  cudaStream_t to enqueue on (NULL: the legacy default stream).
 * Asynchronous: the value is in `out` once the stream reaches it.  Scratch
 * is a file-scope device array of 65536 doubles (512 KiB) that every GPU
 * loading the library holds until exit, so lattices above 8,388,608 sites
 * fail with YM_ERR_SCRATCH_TOO_SMALL before any device work.  All calls
 * share that array: calls that overlap on the GPU (concurrent streams or
 * threads) race and must be serialised by the caller.  The first call on a
 * device resolves the array's device address for that device (and the first
 * call after a device reset resolves it again); make that first call before
 * any stream capture.  A CUDA failure returns YM_ERR_CUDA with the error
 * readable through ym_last_cuda_error. */
int32_t ym_su3_average_plaquette_noalloc(const double *links, const int64_t *extents,
                                         double *out, void *stream);

/* Lattice-averaged rectangular Wilson loops: for every chain, every plane
 * (mu < nu) in the order (0,1),(0,2),(0,3),(1,2),(1,3),(2,3) and every
 * R <= rmax, T <= tmax (both in 1..4) the mean over start sites of
 * Re wilson_loop(x, rectangular_path(mu, nu, R, T)) (path_holonomy.rs:172-260;
 * R steps along mu, T along nu).  out[((chain*6 + plane)*4 + R-1)*4 + T-1];
 * entries beyond (rmax, tmax) are 0.  The lattice average has no reference
 * counterpart; each per-site value is the reference's primitive, evaluated
 * as Re Tr of the closed path's two halves (agreeing with the reference's
 * single left-to-right product to rounding; means within 1e-12). */
int32_t ym_su3_wilson_loops(ym_ensemble *ens, int32_t rmax, int32_t tmax, double *out);
/* Polyakov loop (su3_lattice.rs:185-212) averaged over every start site with
 * x_dir = 0: out[chain*2 + 0] = mean Re, out[chain*2 + 1] = mean Im. */
int32_t ym_su3_polyakov_loops(ym_ensemble *ens, int32_t direction, double *out);
/* SU(2) lattice averages of the reference's loops: for every chain, plane
 * and R <= rmax, T <= tmax (1..4) the mean over start sites of
 * Lattice4::rectangular_wilson_loop(x, mu, nu, R, T) (lib.rs:471-481, the
 * single left-to-right product of rectangular_path's steps, half real
 * trace), laid out as ym_su3_wilson_loops; and the mean over the lines along
 * `direction` of Lattice4::polyakov_loop (lib.rs:483-505), one double per
 * chain.  The lattice averages have no reference counterpart; each per-site
 * value is the reference's primitive with its arithmetic. */
int32_t ym_su2_wilson_loops(ym_ensemble *ens, int32_t rmax, int32_t tmax, double *out);
int32_t ym_su2_polyakov_loops(ym_ensemble *ens, int32_t direction, double *out);

/* ---- per-site and per-link queries (Su3Lattice4, Lattice4, path_holonomy)
 * on binary64 handles of either group.  Sites are given as 4 coordinates
 * (x0, x1, x2, x3) and per-site outputs are in the reference's lexicographic
 * site order (x3 fastest).  A path is a list of steps: +(d+1) steps forward
 * along direction d, -(d+1) backward (path_holonomy::OrientedStep,
 * lib.rs PathStep).  SU(3) products are the reference's checked products
 * (Su3::mul su3.rs:286-288): a product outside the 5e-12 group gates fails
 * with YM_ERR_NON_FINITE_MATRIX / YM_ERR_NON_UNITARY_MATRIX /
 * YM_ERR_DETERMINANT_NOT_ONE.  Every value below is bit for bit the
 * reference's arithmetic in the reference's order. ---- */

/* path_holonomy::rectangular_path (path_holonomy.rs:219-260; lib.rs:438-469):
 * R steps forward along mu, T forward along nu, R back, T back.  steps has
 * room for `capacity` entries; *n_steps = 2(R+T). */
int32_t ym_rectangular_path(int32_t mu, int32_t nu, int64_t r, int64_t t, int32_t *steps,
                            int64_t capacity, int64_t *n_steps);
/* path_holonomy (path_holonomy.rs:132-161; Lattice4::path_holonomy
 * lib.rs:384-414): the ordered product along `steps` from `start` (18 doubles
 * SU(3), 4 doubles SU(2)); end (optional) receives the final site. */
int32_t ym_path_holonomy(ym_ensemble *ens, int64_t chain, const int64_t *start,
                         const int32_t *steps, int64_t n_steps, double *holonomy, int64_t *end);
/* wilson_loop (path_holonomy.rs:172-181: (1/3) Tr of the closed holonomy,
 * complex; Lattice4::wilson_loop lib.rs:430-436: (1/2) Re Tr, imaginary part
 * 0) at one start (out2 = re, im) or from every site of the chain
 * (out[2*lex], out[2*lex+1]).  An open path fails with
 * YM_ERR_PATH_NOT_CLOSED. */
int32_t ym_wilson_loop(ym_ensemble *ens, int64_t chain, const int64_t *start, const int32_t *steps,
                       int64_t n_steps, double *out2);
int32_t ym_wilson_loop_sites(ym_ensemble *ens, int64_t chain, const int32_t *steps, int64_t n_steps,
                             double *out);
/* Su3Lattice4::polyakov_loop(start, direction) (su3_lattice.rs:185-212,
 * complex (1/3) Tr) / Lattice4::polyakov_loop (lib.rs:483-505, (1/2) Re Tr,
 * imaginary part 0) at one start or from every site. */
int32_t ym_polyakov_loop(ym_ensemble *ens, int64_t chain, const int64_t *start, int32_t direction,
                         double *out2);
int32_t ym_polyakov_loop_sites(ym_ensemble *ens, int64_t chain, int32_t direction, double *out);
/* plaquette(x, mu, nu) (su3_lattice.rs:168-181: the SU(3) matrix, 18
 * doubles; lib.rs:348-361: the SU(2) quaternion, 4 doubles). */
int32_t ym_plaquette(ym_ensemble *ens, int64_t chain, const int64_t *x, int32_t mu, int32_t nu,
                     double *out);
/* wilson_action(beta) per chain (su3_lattice.rs:214-242: beta * sum of
 * 1 - (1/3) Re Tr P; lib.rs:363-382: beta * sum of 1 - (1/2) Re Tr P), the
 * terms summed in the reference's sequential order. */
int32_t ym_wilson_action(ym_ensemble *ens, double beta, double *per_chain);
/* Lattice4::staple (lib.rs:507-546): the unnormalised sum of the six staple
 * products of link (x, mu), 4 components; *terms = 6. */
int32_t ym_su2_staple(ym_ensemble *ens, int64_t chain, const int64_t *x, int32_t mu, double *comp4,
                      int64_t *terms);
/* local_link_action (su3_ensemble.rs:311-317) and local_action_difference
 * (su3_ensemble.rs:319-334) of link (x, mu): beta times the sum over the six
 * forward and six backward plaquettes holding the link of
 * 1 - (1/3) Re Tr P; the difference between the candidate (18 doubles) and
 * the stored link.  beta in [0, 12]. */
int32_t ym_su3_local_link_action(ym_ensemble *ens, int64_t chain, const int64_t *x, int32_t mu,
                                 double beta, double *out);
int32_t ym_su3_local_action_difference(ym_ensemble *ens, int64_t chain, const int64_t *x,
                                       int32_t mu, const double *candidate, double beta,
                                       double *out);
/* Su3Lattice4::gauge_transform (su3_lattice.rs:244-283): chain dst_chain of
 * dst (same extents; dst may be src) receives g(x) U_mu(x) g(x+mu)^dag for
 * every link of chain `chain` of src, each product checked.  site_gauges is a
 * host array of V SU(3) matrices (18 doubles each) in lexicographic site
 * order: the reference's closure evaluated at every site. */
int32_t ym_su3_gauge_transform(ym_ensemble *src, int64_t chain, const double *site_gauges,
                               ym_ensemble *dst, int64_t dst_chain);
/* Su3Lattice4::link / set_link (su3_lattice.rs:153-166), Lattice4::link /
 * set_link: one link (18 doubles SU(3), 4 SU(2)) moved between the host and
 * the device without touching the rest of the chain.  On two-row binary32
 * handles link() returns the binary64 image (third row rebuilt) and
 * set_link() stores the first two rows rounded to binary32. */
int32_t ym_ensemble_get_link(ym_ensemble *ens, int64_t chain, const int64_t *x, int32_t mu,
                             double *out);
int32_t ym_ensemble_set_link(ym_ensemble *ens, int64_t chain, const int64_t *x, int32_t mu,
                             const double *value);

/* scalar_a1pp_operator_basis (glueball_operators.rs:93-160) for every time
 * slice of every chain: the mean of Re W over the three 1x1 and the six 2x1
 * spatial orientations and all spatial start sites.  Outputs packed chain by
 * chain, t = 0..N3-1 (sum over chains of N3 entries each); loop counts are
 * 3 Vs and 6 Vs.  Needs cubic spatial extents >= 3. */
int32_t ym_su3_scalar_operator_basis(ym_ensemble *ens, double *plaquette, double *rectangle);

/* ---- transformations between handles of matching geometry ---- */
int32_t ym_ensemble_copy(ym_ensemble *src, ym_ensemble *dst);
/* Copy one chain's links into a chain of equal extents, group and precision
 * of another handle (device to device). */
int32_t ym_ensemble_copy_chain(ym_ensemble *src, int64_t src_chain, ym_ensemble *dst,
                               int64_t dst_chain);
/* The same for `count` consecutive chains (src_first.. into dst_first..),
 * each pair of equal extents: chains of a handle are laid out back to back,
 * so this is one device-to-device copy and one synchronisation. */
int32_t ym_ensemble_copy_chains(ym_ensemble *src, int64_t src_first, ym_ensemble *dst,
                                int64_t dst_first, int64_t count);
/* spatial_stout_smear (glueball_smearing.rs:257-268): `levels` synchronous
 * spatial stout levels of src written to dst (same extents); rho in
 * (0, 0.25], levels <= 8 unless lift_level_cap (sequential levels compose,
 * so 10 = 8 then 2 exactly).  dst may be src (smearing in place, so a
 * caller measuring after 0, 5 and 10 levels smears 5 + 5, not 15). */
int32_t ym_su3_spatial_stout_smear(ym_ensemble *src, ym_ensemble *dst, double rho, int64_t levels,
                                   int32_t lift_level_cap);
/* spatial_stride2_block (glueball_blocking.rs:105-136): dst holds the
 * blocked extents (N0/2, N1/2, N2/2, N3) of every src chain. */
int32_t ym_su3_spatial_stride2_block(ym_ensemble *src, ym_ensemble *dst);

/* One measurement of the scalar-glueball production cadence
 * (glueball_scalar_production.rs:257-381, per retained configuration): the
 * links of `ens` copied into `smeared` (same extents), then for each stout
 * level count in `levels` (ascending; 0 allowed) the levels smeared
 * continuing from the previous count (sequential levels, so the same links
 * as smearing from scratch; spatial_stout_smear glueball_smearing.rs:257;
 * on return `smeared` holds the last level),
 * scalar_a1pp_operator_basis of every chain (glueball_operators.rs:93-160),
 * and for every blocked group g the chains first_chain[g].. of `smeared`
 * copied into fine[g], spatial_stride2_block into coarse[g]
 * (glueball_blocking.rs:105-136) and its operator basis.  The whole
 * measurement is one captured CUDA graph, replayed on later calls with the
 * same plan and handles, with a single synchronisation at the end.
 *   plaquette, rectangle          [n_levels][slices of smeared]
 *   blocked_plaquette, _rectangle [n_levels][slices of coarse[0], coarse[1], ...]
 * (slices: every chain's time slices t = 0..N3-1, chain by chain, as
 * ym_su3_scalar_operator_basis returns them). */
typedef struct {
    double rho;                      /* (0, 0.25] */
    int32_t n_levels;
    const int64_t *levels;
    int32_t n_blocked;
    ym_ensemble *const *fine;        /* n_blocked handles */
    ym_ensemble *const *coarse;      /* n_blocked handles of the blocked extents */
    const int64_t *first_chain;      /* n_blocked */
} ym_glueball_plan;
int32_t ym_su3_glueball_measure(ym_ensemble *ens, ym_ensemble *smeared, const ym_glueball_plan *plan,
                                double *plaquette, double *rectangle, double *blocked_plaquette,
                                double *blocked_rectangle);
/* The set-up half of ym_su3_glueball_measure (no reference counterpart):
 * validates the plan, allocates the handles' scratch, captures the
 * measurement graph and uploads it, without measuring; a later
 * ym_su3_glueball_measure with the same plan and handles only launches it.
 * Production drivers call it once before their first measurement. */
int32_t ym_su3_glueball_prepare(ym_ensemble *ens, ym_ensemble *smeared, const ym_glueball_plan *plan);

/* ---- two-row binary32 storage (YM_PREC_F32_TWO_ROW, no reference
 * counterpart: the reference stores 18 doubles per link) ----
 * Gram-Schmidt of every link's two stored rows in binary64, rounded back;
 * the third row is always rebuilt as conj(row0 x row1).  Every sweep of a
 * two-row handle ends with this step (the representation is unstable
 * without it); a caller needs it only after uploading foreign links. */
int32_t ym_su3_reunitarize(ym_ensemble *ens);
/* Copy src into dst of the same extents, converting between YM_PREC_F64 and
 * YM_PREC_F32_TWO_ROW (binary64 third row rebuilt from the stored rows).
 * Observables other than the plaquette read binary64 handles; a two-row
 * chain is measured through such a converted copy. */
int32_t ym_ensemble_convert(ym_ensemble *src, ym_ensemble *dst);

/* ---- connected correlators (host FP64, the reference's order) ----
 * samples are [configuration][time].
 * periodic_connected_estimator (glueball_correlators.rs:111-172). */
int32_t ym_periodic_connected_estimator(const double *samples, int64_t n_configurations,
                                        int64_t time_extent, double *vacuum_mean, double *raw,
                                        double *connected);
/* connected_from_samples (glueball_scalar_production.rs:383-443); omitted < 0
 * keeps every configuration. */
int32_t ym_connected_from_samples(const double *samples, int64_t n_configurations,
                                  int64_t time_extent, int64_t omitted, double *connected);
/* All delete-one jackknife replicas: replicas[k][tau] = connected_from_samples
 * omitting configuration k. */
int32_t ym_jackknife_replicas(const double *samples, int64_t n_configurations, int64_t time_extent,
                              double *replicas);
/* jackknife_covariance (glueball_scalar_fit.rs:276-322) over the window
 * [start, end]; out is (end-start+1)^2 row-major. */
int32_t ym_jackknife_covariance(const double *replicas, int64_t n_replicas, int64_t time_extent,
                                int64_t start, int64_t end, double *out);

/* Largest unitarity and determinant residual per chain
 * (Su3Lattice4::max_link_*_residual su3_lattice.rs:285-297). */
int32_t ym_su3_max_residuals(ym_ensemble *ens, double *unitarity, double *determinant);

/* ---- host-side FP64 analysis and stream helpers ---- */

/* ChainDiagnostics (su2_ensemble.rs:161-170); the autocorrelation series is
 * written to a caller array of max_lag+1 doubles. */
typedef struct {
    double mean;
    double variance;
    int64_t positive_window_lag;
    double integrated_autocorrelation_time;
    double effective_sample_size;
    double standard_error;
} ym_chain_diagnostics;

/* EfficiencyReport (sampling_efficiency.rs:22-34). */
typedef struct {
    ym_chain_diagnostics diagnostics;
    double reweighting_efficiency;
    double weight_only_ess;
    double combined_ess_proxy;
    double total_cost;
    double sampling_cost_per_effective_sample_proxy;
    double total_cost_per_effective_sample_proxy;
} ym_efficiency_report;

/* derive_chain_seed (su2_ensemble.rs:52-55) and derive_su3_chain_seed
 * (su3_ensemble.rs:189-192). */
uint64_t ym_derive_chain_seed(uint64_t master_seed, uint64_t chain_id);
uint64_t ym_derive_su3_chain_seed(uint64_t master_seed, uint64_t chain_id);
/* Output n (0-based) of SplitMix64::new(seed) (su2_ensemble.rs:29-37). */
uint64_t ym_splitmix64_at(uint64_t seed, uint64_t n);
/* proposal_angle_from_u64 (su3_ensemble.rs:199-213). */
int32_t ym_proposal_angle_from_u64(uint64_t raw, double proposal_angle, double *out);
/* diagnostics (su2_ensemble.rs:375-463). */
int32_t ym_diagnostics(const double *values, int64_t n, int64_t max_lag,
                       ym_chain_diagnostics *out, double *autocorrelation);
/* evaluate (sampling_efficiency.rs:57-135); log_weights may be NULL. */
int32_t ym_sampling_efficiency(const double *values, int64_t n, const double *log_weights,
                               int64_t max_lag, double setup, double thermalization,
                               double sampling, ym_efficiency_report *out,
                               double *autocorrelation);

/* ---- kernel timing (no reference counterpart: the reference counts cost in
 * proposals only) ----  While enabled, each launch of the listed kernels is
 * bracketed by CUDA events on the handle's stream; ym_profile_read
 * synchronises, returns the summed device time and launch count of one
 * kernel since the last read, and resets it.  YM_KERNEL_AUX covers the
 * Wilson-loop and Polyakov-loop measurements (one bracket per call). */
enum { YM_KERNEL_SU3_METROPOLIS = 0, YM_KERNEL_PLAQUETTE = 1, YM_KERNEL_SU2_HEATBATH = 2,
       YM_KERNEL_SU2_OVERRELAX = 3, YM_KERNEL_STOUT = 4, YM_KERNEL_OPERATORS = 5,
       YM_KERNEL_AUX = 6, YM_KERNEL_LEARNED = 7, YM_KERNEL_COUNT = 8 };
int32_t ym_profile_enable(ym_ensemble *ens, int32_t on);
int32_t ym_profile_read(ym_ensemble *ens, int32_t kernel, double *total_ms, int64_t *launches);

/* Per-chain coupling and stream seed (the reference passes beta and the
 * stream to every sweep call, su3_ensemble.rs:342-347). */
int32_t ym_ensemble_set_chain(ym_ensemble *ens, int64_t chain, double beta, uint64_t chain_seed);

#ifdef __cplusplus
}
#endif

#endif /* YMGPU_H */
