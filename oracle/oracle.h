/* oracle.h -- public entry points of the CPU oracle (liboracle.so).
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference crate
 * (QSOLKCB/YANG-MILLS) used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py to check the CUDA engine.  Nothing in the
 * product links it.  Every function returns a ym_status code.
 *
 * Lattices are caller-owned arrays in the reference's memory order:
 * link index = site*4 + mu with site = ((x0*N1 + x1)*N2 + x2)*N3 + x3;
 * SU(3) links are 18 doubles (3x3 row-major, re/im interleaved), SU(2)
 * links 4 doubles (unit quaternion).
 */
#ifndef YM_ORACLE_H
#define YM_ORACLE_H

#include <stdint.h>

#include "../include/ym_status.h"

typedef struct {
    int64_t extents[4];
    double beta;
    uint64_t master_seed;
    uint64_t chain_id;
    int64_t thermalization_sweeps;
    int64_t measurements;
    int64_t sweeps_between_measurements;
    double proposal_angle;
    int64_t autocorrelation_max_lag;
} or_su3_config;

typedef struct {
    uint64_t derived_seed;
    int64_t total_sweeps;
    uint64_t proposals;
    uint64_t accepts;
    double mean_acceptance;
    double final_unitarity_residual;
    double final_determinant_residual;
} or_su3_chain_scalars;

typedef struct {
    int64_t extents[4];
    double beta;
    uint64_t master_seed;
    uint64_t chain_id;
    int64_t thermalization_sweeps;
    int64_t measurements;
    int64_t sweeps_between_measurements;
    int64_t overrelaxation_sweeps_per_heatbath;
    int64_t max_heatbath_attempts_per_link;
    int64_t autocorrelation_max_lag;
} or_su2_config;

typedef struct {
    uint64_t derived_seed;
    int64_t total_heatbath_sweeps;
    int64_t total_overrelaxation_sweeps;
    uint64_t heatbath_proposals;
    uint64_t heatbath_updates;
    double mean_heatbath_acceptance;
    double final_link_unit_residual;
} or_su2_chain_scalars;

typedef struct {
    double mean;
    double variance;
    int64_t positive_window_lag;
    double integrated_autocorrelation_time;
    double effective_sample_size;
    double standard_error;
} or_diagnostics_out;

typedef struct {
    or_diagnostics_out diagnostics;
    double reweighting_efficiency;
    double weight_only_ess;
    double combined_ess_proxy;
    double total_cost;
    double sampling_cost_per_effective_sample_proxy;
    double total_cost_per_effective_sample_proxy;
} or_efficiency_out;

/* SplitMix64 / seeds (su2_ensemble.rs:24-55, su3_ensemble.rs:183-192) */
uint64_t or_mix64_pub(uint64_t v);
uint64_t or_splitmix_next(uint64_t *state);
double or_splitmix_unit(uint64_t *state);
uint64_t or_derive_chain_seed(uint64_t master, uint64_t chain);
uint64_t or_derive_su3_chain_seed(uint64_t master, uint64_t chain);
int or_proposal_angle_from_u64(uint64_t raw, double angle, double *out);

/* SU(2) (lib.rs, su2_ensemble.rs) */
int or_su2_mul(const double *a, const double *b, double *out);
int or_su2_from_axis_angle(const double *axis, double angle, double *out);
int or_su2_from_normalized(const double *c, double *out);
int or_su2_identity(const int64_t *ext, double *links);
int or_su2_plaquette(const int64_t *ext, const double *links, const int64_t *x, int mu, int nu,
                     double *out4);
int or_su2_wilson_action(const int64_t *ext, const double *links, double beta, double *out);
int or_su2_wilson_loop(const int64_t *ext, const double *links, const int64_t *start,
                       const int32_t *steps, int64_t nsteps, double *out);
int or_su2_polyakov_loop(const int64_t *ext, const double *links, const int64_t *start, int dir,
                         double *out);
int or_su2_staple(const int64_t *ext, const double *links, const int64_t *x, int mu, double *out4);
int or_su2_max_unit_residual(const int64_t *ext, const double *links, double *out);
int or_su2_sample_heatbath(double alpha, uint64_t *rng, int64_t max_attempts, double *out4,
                           uint64_t *attempts);
int or_su2_heatbath_sweep(const int64_t *ext, double *links, double beta, uint64_t *rng,
                          int64_t max_attempts, uint64_t *proposals, uint64_t *updates);
int or_su2_overrelaxation_sweep(const int64_t *ext, double *links);
int or_su2_average_plaquette(const int64_t *ext, const double *links, double *out);
int or_su2_run_chain(const or_su2_config *cfg, double *links_out, double *measurements,
                     or_su2_chain_scalars *out);
/* Engine update order (checkerboard, per-link counter streams). */
int or_su2_cb_sweep(const int64_t *ext, double *links, double beta, uint64_t chain_seed,
                    uint64_t sweep, int64_t overrelaxation_sweeps, int64_t max_attempts,
                    uint64_t *proposals);

/* SU(3) (su3.rs, su3_lattice.rs, path_holonomy.rs, su3_ensemble.rs) */
int or_su3_identity(const int64_t *ext, int lift_cap, double *links);
int or_su3_from_algebra(const double *coef, double *out18);
int or_su3_mul(const double *a18, const double *b18, double *out18);
int or_su3_matrix_residuals(const double *m18, double *unitarity, double *determinant);
int or_su3_structure(int a, int b, int c, double *f, double *d);
int or_su3_plaquette_matrix(const int64_t *ext, const double *links, const int64_t *x, int mu,
                            int nu, double *out18);
int or_su3_wilson_action(const int64_t *ext, const double *links, double beta, double *out);
int or_su3_polyakov_loop(const int64_t *ext, const double *links, const int64_t *start, int dir,
                         double *out_re, double *out_im);
int or_su3_gauge_transform(const int64_t *ext, const double *links, const double *site_gauges,
                           double *out_links);
int or_su3_max_residuals(const int64_t *ext, const double *links, double *unitarity,
                         double *determinant);
int or_su3_traceless_cycle_link(double *out18);
int or_su3_deterministic_site_gauge(const int64_t *x, double *out18);
int or_su3_path_holonomy(const int64_t *ext, const double *links, const int64_t *start,
                         const int32_t *steps, int64_t nsteps, double *out18, int64_t *end);
int or_rectangular_path(int mu, int nu, int64_t r, int64_t t, int32_t *steps, int64_t cap,
                        int64_t *n);
int or_su3_wilson_loop(const int64_t *ext, const double *links, const int64_t *start,
                       const int32_t *steps, int64_t nsteps, double *re, double *im);
int or_su3_average_plaquette(const int64_t *ext, const double *links, double *out);
int or_su3_local_action_difference(const int64_t *ext, const double *links, const int64_t *x,
                                   int mu, const double *cand18, double beta, double *out);
int or_su3_metropolis_sweep(const int64_t *ext, double *links, double beta, double angle,
                            uint64_t *rng, uint64_t *proposals, uint64_t *accepts);
int or_su3_run_chain(const or_su3_config *cfg, double *links_out, double *measurements,
                     or_su3_chain_scalars *out);

/* Statistics (su2_ensemble.rs:375-463, sampling_efficiency.rs,
 * glueball_correlators.rs, glueball_scalar_production.rs, glueball_scalar_fit.rs) */
int or_diagnostics(const double *v, int64_t n, int64_t max_lag, or_diagnostics_out *o,
                   double *autocorrelation);
int or_sampling_efficiency(const double *v, int64_t n, const double *log_weights, int64_t max_lag,
                           double setup, double thermalization, double sampling,
                           or_efficiency_out *o, double *autocorrelation);
int or_periodic_connected_estimator(const double *samples, int64_t ncfg, int64_t nt,
                                    double *vacuum_mean, double *raw, double *connected);
int or_connected_from_samples(const double *samples, int64_t ncfg, int64_t nt, int64_t omitted,
                              double *connected);
int or_jackknife_covariance(const double *replicas, int64_t nrep, int64_t nt, int64_t start,
                            int64_t end, double *out);

/* Glueball transformations and operators */
int or_scalar_a1pp_operator_basis(const int64_t *ext, const double *links, int64_t t,
                                  double *plaq, double *rect, int64_t *plaq_count,
                                  int64_t *rect_count);
int or_spatial_stout_smear(const int64_t *ext, const double *links, double rho, int64_t levels,
                           int lift_level_cap, double *out);
int or_max_link_residual(const int64_t *ext, const double *a, const double *b, double *out);
int or_blocked_extents(const int64_t *ext, int64_t *out);
int or_spatial_stride2_block(const int64_t *ext, const double *links, double *coarse);
int or_scalar_connected_correlators(const int64_t *ext, const double *configs, int64_t ncfg,
                                    double *vac, double *raw, double *connected);

/* Engine update order restated on the CPU (or_b200.c) */
uint64_t or_splitmix_at(uint64_t seed, uint64_t n);
uint64_t or_cb_link_key(uint64_t chain_seed, uint64_t sweep, int64_t lex, int mu);
int or_su3_generator_rotation(int g, double theta, double *out18);
int or_su3_staple(const int64_t *ext, const double *links, const int64_t *x, int mu, double *out18);
int or_su3_visit(double *u18, const double *a18, double beta, double angle, uint64_t key,
                 int uniform_generator, uint64_t *accepts);
int or_su3_cb_sweep(const int64_t *ext, double *links, double beta, double angle,
                    uint64_t chain_seed, uint64_t sweep, int uniform_generator,
                    uint64_t *proposals, uint64_t *accepts);
int or_su3_plaquette_value(const int64_t *ext, const double *links, const int64_t *x, int mu,
                           int nu, double *out);
int or_su3_hit(double *u18, const double *a18, double beta, double angle, uint64_t w_angle,
               uint64_t w_acc, int g, uint64_t *accepted);

/* Learned proposal (or_learned.c) */
float or_bf16_round(float x);
int or_lp_features(const double *a18, double beta, double *f16);
int or_lp_forward(const float *params, const float *x, int64_t n, double *y);
int or_lp_proposal(const double *y16, double *p8, double *scale);
int or_lp_objective(const double *y16, const float *m18, double beta, double *e_out, double *dy9);
int or_lp_loss_grad(const float *params, const float *x, const float *m18, const double *beta,
                    int64_t n, double *objective, double *grad);
int or_lp_loss_grad_mode(const float *params, const float *x, const float *m18,
                         const double *beta, int64_t n, int exact, double *objective,
                         double *grad);
int or_lp_retr_rotated(int g, const float *m18, double theta, double *f, double *df);
int or_lp_objective_exact(const double *params, const double *x, const float *m18,
                          const double *beta, int64_t n, double *objective);
int or_lp_pick_generator(uint64_t w, const double *p8);
int or_lp_cb_sweep(const int64_t *ext, double *links, double beta, const float *params,
                   uint64_t chain_seed, uint64_t sweep, uint64_t *proposals, uint64_t *accepts);

/* Multi-threaded CPU baseline of the reference Metropolis sweep (or_threads.c) */
int or_bench_su3_reference(const int64_t *ext, double beta, double angle, uint64_t master_seed,
                           int64_t threads, int64_t links_per_thread, double *seconds,
                           uint64_t *link_updates);

#endif /* YM_ORACLE_H */
