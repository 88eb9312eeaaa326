/* ym_analysis.h -- host FP64 analysis of glueball correlators: cosh
 * effective mass with jackknife errors, the correlated single-state fit,
 * and the two-operator variational (GEVP) projection.
 *
 * These replace the reference's module-level Rust functions one for one
 * (QSOLKCB/YANG-MILLS, reference/rust/src):
 *   ym_cosh_effective_mass_with_jackknife  glueball_effective_mass.rs:170
 *   ym_analytic_periodic_single_state      glueball_effective_mass.rs:237
 *   ym_correlated_scalar_fit               glueball_scalar_fit.rs:595
 *   ym_canonical_scalar_fit_fixture        glueball_scalar_fit.rs:663
 *   ym_scalar_variational_connected_correlator
 *                                          glueball_scalar_variational.rs:628
 *   ym_principal_generalized_projection    glueball_scalar_variational.rs:746
 *   ym_canonical_two_state_matrices        glueball_scalar_variational.rs:931
 *   ym_max_matrix_series_residual          glueball_scalar_variational.rs:953
 * plus three of the fit's private steps that the reference's tests call
 * directly (jackknife_covariance :276, invert_matrix :361,
 * maximum_off_diagonal_correlation :567).
 *
 * A jackknife replica set is the reference's &[Vec<f64>]: an array of
 * n_replicas row pointers and their lengths (a ragged set is what
 * ShapeMismatch rejects).  Lags and window bounds are usize in the
 * reference and uint64_t here.  A 2x2 correlator matrix series is
 * [time][row][column], row-major.  The variational correlator takes the
 * per-slice operator samples [configuration][time][2] (plaquette 1x1,
 * rectangle 2x1) that ym_a1pp_operator_basis produces on the device, where
 * the reference evaluates them from each configuration.  Failures are the
 * reference's variants (ym_status.h), checked in the reference's order.
 */
#ifndef YM_ANALYSIS_H
#define YM_ANALYSIS_H

#include <stdint.h>

#include "ym_status.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t tau;
    double full_estimate;
    double jackknife_mean;
    double standard_error;
} ym_effective_mass_point;

/* points[n_lags] receives one point per lag. */
int32_t ym_cosh_effective_mass_with_jackknife(const double *full, int64_t time_extent,
                                              const double *const *jackknife,
                                              const int64_t *jackknife_lengths, int64_t n_replicas,
                                              const uint64_t *lags, int64_t n_lags,
                                              ym_effective_mass_point *points);
/* C(tau) = A (exp(-m tau) + exp(-m (N_t - tau))), tau = 0..N_t-1. */
int32_t ym_analytic_periodic_single_state(int64_t time_extent, double mass, double amplitude,
                                          double *correlator);

typedef struct {
    uint64_t start;
    uint64_t end; /* inclusive */
} ym_fit_window;

typedef struct {
    int64_t time_extent;
    int64_t jackknife_replicates;
    ym_fit_window selected_window;
    double plateau_weighted_effective_mass;
    double plateau_maximum_z;
    double fitted_mass;
    double fitted_amplitude;
    double chi_square;
    int64_t degrees_of_freedom;
    double chi_square_per_dof;
    double mass_jackknife_mean;
    double mass_standard_error;
    double amplitude_jackknife_mean;
    double amplitude_standard_error;
    double maximum_off_diagonal_correlation;
} ym_scalar_fit_result;

int32_t ym_correlated_scalar_fit(const double *full, int64_t time_extent,
                                 const double *const *jackknife, const int64_t *jackknife_lengths,
                                 int64_t n_replicas, const ym_fit_window *candidates,
                                 int64_t n_candidates, ym_scalar_fit_result *result);
/* covariance[p][p], p = window points. */
int32_t ym_scalar_fit_window_covariance(const double *const *jackknife,
                                        const int64_t *jackknife_lengths, int64_t n_replicas,
                                        ym_fit_window window, double *covariance);
int32_t ym_scalar_fit_invert_covariance(const double *matrix, int64_t n, double *inverse);
int32_t ym_maximum_off_diagonal_correlation(const double *covariance, int64_t n, double *out);
/* full[16], jackknife[8][16], candidates[3]. */
int32_t ym_canonical_scalar_fit_fixture(double *full, double *jackknife, ym_fit_window *candidates);

typedef struct {
    int64_t reference_time;
    int64_t diagonalization_time;
    double principal_eigenvalue;
    double coefficients[2];
} ym_principal_projection;

/* samples[n_configurations][time_extent][2] -> vacuum_means[2],
 * matrices[time_extent][2][2]. */
int32_t ym_scalar_variational_connected_correlator(const double *samples, int64_t n_configurations,
                                                   int64_t time_extent, double *vacuum_means,
                                                   double *matrices);
/* projected[time_extent] receives v^T C(t) v for the principal vector v. */
int32_t ym_principal_generalized_projection(const double *matrices, int64_t time_extent,
                                            int64_t reference_time, int64_t diagonalization_time,
                                            ym_principal_projection *result, double *projected);
/* matrices[16][2][2]. */
int32_t ym_canonical_two_state_matrices(double *matrices);
int32_t ym_max_matrix_series_residual(const double *first, int64_t n_first, const double *second,
                                      int64_t n_second, double *out);

#ifdef __cplusplus
}
#endif

#endif /* YM_ANALYSIS_H */
