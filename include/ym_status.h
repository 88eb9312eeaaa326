/* ym_status.h -- status codes shared by every entry point of libymgpu.
 *
 * The reference library (QSOLKCB/YANG-MILLS, Rust) reports failures through
 * nested fail-closed `Result` enums.  Across a C ABI those become one flat
 * int32 namespace: 0 is success and every other value names exactly one
 * innermost reference variant (nested wrappers such as
 * `Su3EnsembleError::Lattice(Su3LatticeError::X)` map to the code of `X`).
 * The enum each block mirrors is cited beside it.  Codes >= 900 have no
 * reference counterpart: they describe the device boundary itself.
 */
#ifndef YM_STATUS_H
#define YM_STATUS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ym_status {
    YM_OK = 0,

    /* ReferenceError (reference/rust/src/lib.rs:52-73) and
     * Su3LatticeError (reference/rust/src/su3_lattice.rs:26-39). */
    YM_ERR_NON_FINITE_SU2_COMPONENT = 1,
    YM_ERR_ZERO_SU2_NORM = 2,
    YM_ERR_NON_UNIT_SU2 = 3,
    YM_ERR_INVALID_AXIS = 4,
    YM_ERR_INVALID_LATTICE_EXTENT = 5,
    YM_ERR_LATTICE_SIZE_OVERFLOW = 6,
    YM_ERR_LATTICE_TOO_LARGE = 7,
    YM_ERR_ALLOCATION_FAILED = 8,
    YM_ERR_COORDINATE_OUT_OF_RANGE = 9,
    YM_ERR_DIRECTION_OUT_OF_RANGE = 10,
    YM_ERR_DIRECTIONS_MUST_DIFFER = 11,
    YM_ERR_NON_FINITE_BETA = 12,
    YM_ERR_NEGATIVE_BETA = 13,
    YM_ERR_NON_FINITE_ACTION = 14,
    YM_ERR_EMPTY_PATH = 15,
    YM_ERR_PATH_TOO_LONG = 16,
    YM_ERR_PATH_NOT_CLOSED = 17,
    YM_ERR_ZERO_RECTANGLE_EXTENT = 18,
    YM_ERR_INVALID_CONFIGURATION_ENCODING = 19,

    /* EnsembleError (reference/rust/src/su2_ensemble.rs:109-121). */
    YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE = 30,
    YM_ERR_SCHEDULE_OUTSIDE_REFERENCE_RANGE = 31,
    YM_ERR_TOO_FEW_MEASUREMENTS = 32,
    YM_ERR_ZERO_MEASUREMENT_STRIDE = 33,
    YM_ERR_TOO_MANY_OVERRELAXATION_SWEEPS = 34,
    YM_ERR_ZERO_HEATBATH_ATTEMPT_LIMIT = 35,
    YM_ERR_AUTOCORRELATION_LAG_OUT_OF_RANGE = 36,
    YM_ERR_HEATBATH_ATTEMPT_LIMIT_EXCEEDED = 37,
    YM_ERR_NON_FINITE_STATISTIC = 38,

    /* Su3Error (reference/rust/src/su3.rs:291-300). */
    YM_ERR_GENERATOR_INDEX_OUT_OF_RANGE = 50,
    YM_ERR_NON_FINITE_COEFFICIENT = 51,
    YM_ERR_ALGEBRA_COEFFICIENT_TOO_LARGE = 52,
    YM_ERR_NON_FINITE_MATRIX = 53,
    YM_ERR_EXPONENTIAL_SCALING_OVERFLOW = 54,
    YM_ERR_NON_UNITARY_MATRIX = 55,
    YM_ERR_DETERMINANT_NOT_ONE = 56,

    /* Su3EnsembleError (reference/rust/src/su3_ensemble.rs:123-137). */
    YM_ERR_PROPOSAL_ANGLE_OUTSIDE_REFERENCE_RANGE = 70,
    YM_ERR_MEASUREMENT_COUNT_OUTSIDE_REFERENCE_RANGE = 71,
    YM_ERR_LATTICE_OUTSIDE_REFERENCE_RANGE = 72,
    YM_ERR_ACCOUNTING_OVERFLOW = 73,
    YM_ERR_DIAGNOSTIC = 74,

    /* GlueballOperatorError (glueball_operators.rs:36-44),
     * GlueballSmearingError (glueball_smearing.rs:33-44),
     * GlueballBlockingError (glueball_blocking.rs:27-35),
     * GlueballCorrelatorError (glueball_correlators.rs:47-60),
     * ProductionError (glueball_scalar_production.rs:159-172),
     * ScalarFitError (glueball_scalar_fit.rs:67-77). */
    YM_ERR_TIME_SLICE_OUT_OF_RANGE = 90,
    YM_ERR_SPATIAL_EXTENT_TOO_SMALL = 91,
    YM_ERR_SPATIAL_EXTENTS_NOT_CUBIC = 92,
    YM_ERR_COUNT_OVERFLOW = 93,
    YM_ERR_NON_FINITE_OBSERVABLE = 94,
    YM_ERR_NON_FINITE_RHO = 95,
    YM_ERR_RHO_OUT_OF_RANGE = 96,
    YM_ERR_TOO_MANY_LEVELS = 97,
    YM_ERR_NON_FINITE_STAPLE = 98,
    YM_ERR_ALGEBRA_PROJECTION_RESIDUAL = 99,
    YM_ERR_SPATIAL_EXTENT_NOT_EVEN = 100,
    YM_ERR_NON_FINITE_RESIDUAL = 101,
    YM_ERR_EMPTY_CONFIGURATION_SET = 102,
    YM_ERR_TOO_MANY_CONFIGURATIONS = 103,
    YM_ERR_TIME_EXTENT_TOO_LARGE = 104,
    YM_ERR_LATTICE_EXTENTS_MISMATCH = 105,
    YM_ERR_SAMPLE_COUNT_OVERFLOW = 106,
    YM_ERR_NON_FINITE_ACCUMULATOR = 107,
    YM_ERR_CORRELATOR_SHAPE_MISMATCH = 108,
    YM_ERR_CONFIGURATION_SHAPE_MISMATCH = 109,
    YM_ERR_INVALID_CANDIDATE_WINDOW = 110,
    YM_ERR_INSUFFICIENT_REPLICATES_FOR_COVARIANCE = 111,

    /* EfficiencyError (reference/rust/src/sampling_efficiency.rs:36-45). */
    YM_ERR_INVALID_LENGTH = 120,
    YM_ERR_INVALID_LAG = 121,
    YM_ERR_INVALID_WEIGHT = 122,
    YM_ERR_INVALID_COST = 123,
    YM_ERR_INVALID_DIAGNOSTIC = 124,
    YM_ERR_DEGENERATE_OBSERVABLE = 125,
    YM_ERR_NON_FINITE_RESULT = 126,

    /* EffectiveMassError (glueball_effective_mass.rs:40-54; TimeExtentTooLarge,
     * NonFiniteStatistic and AllocationFailed share the codes above),
     * ScalarFitError (glueball_scalar_fit.rs:67-81; EffectiveMass(e) is e's
     * code) and VariationalError (glueball_scalar_variational.rs:59-78;
     * Operator(e) and Correlator(e) are e's code). */
    YM_ERR_TIME_EXTENT_TOO_SMALL = 130,
    YM_ERR_TOO_FEW_JACKKNIFE_REPLICATES = 131,
    YM_ERR_TOO_MANY_JACKKNIFE_REPLICATES = 132,
    YM_ERR_EMPTY_ANALYSIS_WINDOW = 133,
    YM_ERR_INVALID_ANALYSIS_LAG = 134,
    YM_ERR_SHAPE_MISMATCH = 135,
    YM_ERR_NON_FINITE_CORRELATOR = 136,
    YM_ERR_NON_POSITIVE_CENTRAL_CORRELATOR = 137,
    YM_ERR_ACOSH_DOMAIN_VIOLATION = 138,
    YM_ERR_INVALID_FIXTURE_PARAMETER = 139,
    YM_ERR_EMPTY_CANDIDATE_WINDOWS = 140,
    YM_ERR_TOO_MANY_CANDIDATE_WINDOWS = 141,
    YM_ERR_DUPLICATE_CANDIDATE_WINDOW = 142,
    YM_ERR_DEGENERATE_PLATEAU_UNCERTAINTY = 143,
    YM_ERR_NO_ACCEPTED_PLATEAU_WINDOW = 144,
    YM_ERR_COVARIANCE_NOT_POSITIVE_DEFINITE = 145,
    YM_ERR_SINGULAR_COVARIANCE = 146,
    YM_ERR_NO_FINITE_GRID_FIT = 147,
    YM_ERR_MATRIX_NOT_SYMMETRIC = 150,
    YM_ERR_INVALID_REFERENCE_TIMES = 151,
    YM_ERR_REFERENCE_MATRIX_NOT_POSITIVE_DEFINITE = 152,
    YM_ERR_DEGENERATE_PRINCIPAL_EIGENVECTOR = 153,
    YM_ERR_NON_POSITIVE_PRINCIPAL_EIGENVALUE = 154,
    YM_ERR_PROJECTION_NORMALIZATION_FAILURE = 155,

    /* BenchmarkError (su2_benchmark.rs:56-66, su3_benchmark.rs:56-66; its
     * NonFiniteStatistic is code 38). */
    YM_ERR_WRONG_BENCHMARK_CONFIGURATION = 160,
    YM_ERR_DUPLICATE_CHAIN_IDENTITY = 161,
    YM_ERR_DUPLICATE_MEASUREMENT_SERIES = 162,
    YM_ERR_INVALID_PLAQUETTE_SAMPLE = 163,
    YM_ERR_INVALID_HEATBATH_ACCOUNTING = 164,
    YM_ERR_INVALID_METROPOLIS_ACCOUNTING = 165,
    YM_ERR_INVALID_ACCEPTANCE_EVIDENCE = 166,
    YM_ERR_INVALID_LINK_UNIT_RESIDUAL = 167,
    YM_ERR_INVALID_LINK_RESIDUAL = 168,
    YM_ERR_STATIONARITY_DIAGNOSTIC_FAILED = 169,

    /* ProductionError (glueball_scalar_production.rs:159-172; its other
     * variants share the codes above or wrap an inner variant). */
    YM_ERR_CORRELATOR_REPLAY_MISMATCH = 170,
    YM_ERR_LINK_RESIDUAL_EXCEEDED = 171,

    /* Device boundary (no reference counterpart). */
    YM_ERR_NULL_ARGUMENT = 900,
    YM_ERR_INVALID_ARGUMENT = 901,
    YM_ERR_CUDA = 902,
    YM_ERR_NOT_CHECKERBOARDABLE = 903, /* a checkerboard sweep needs every extent even */
    YM_ERR_DEVICE_WAIT_TIMEOUT = 904,
    YM_ERR_WRONG_GROUP = 905,          /* handle holds SU(2) where SU(3) was asked, or back */
    YM_ERR_UNSUPPORTED_PRECISION = 906,
    YM_ERR_SCRATCH_TOO_SMALL = 907
} ym_status;

#ifdef __cplusplus
}
#endif

#endif /* YM_STATUS_H */
