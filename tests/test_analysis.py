"""Host analysis of glueball correlators (include/ym_analysis.h) against the
pure-Python oracle and the reference's golden vectors and known answers.

The oracle (oracle/analysis_oracle.py) is pinned to the reference's
test-vectors (glueball-effective-mass-phase3d-v1, glueball-scalar-fit-
phase3e-v1, glueball-scalar-variational-phase3j-v1) and to literal answers
of the reference's unit tests (glueball_effective_mass.rs:265-384,
glueball_scalar_fit.rs:692-813, glueball_scalar_variational.rs:977-1770);
the engine's host functions must equal the oracle bit for bit on seeded
inputs and reproduce every fail-closed variant.  Host code only: no GPU.
"""
import math
import struct

import numpy as np
import pytest

import analysis_oracle as O
from ymgpu import analysis as A
from ymgpu.errors import YmError

MIN_SUBNORMAL = struct.unpack("<d", struct.pack("<Q", 1))[0]
FMAX = 1.7976931348623157e308


def vec(golden, name, vid):
    return [v for v in golden[name]["vectors"] if v["id"] == vid][0]


def variant_of(fn, *args):
    with pytest.raises(YmError) as e:
        fn(*args)
    return e.value.variant


def oracle_variant(fn, *args):
    with pytest.raises(O.AnalysisError) as e:
        fn(*args)
    return e.value.variant


def canonical_em():
    full = A.analytic_periodic_single_state(16, 0.5, 1.0)
    jk = [A.analytic_periodic_single_state(16, m, 1.0) for m in (0.48, 0.49, 0.50, 0.51, 0.52)]
    return full, jk


# ------------------------------------------------------------ phase 3D

def test_effective_mass_golden_oracle_and_engine(golden):
    g = "glueball-effective-mass-phase3d-v1.json"
    v1 = vec(golden, g, "periodic-single-state-cosh-mass")
    v2 = vec(golden, g, "delete-one-jackknife-propagation")
    tol = v1["absolute_tolerance"]
    full = O.analytic_periodic_single_state(v1["time_extent"], v1["full_mass"], v1["amplitude"])
    jk = [O.analytic_periodic_single_state(v1["time_extent"], m, v1["amplitude"])
          for m in v2["replica_masses"]]
    ref = O.cosh_effective_mass_with_jackknife(full, jk, v1["analysis_lags"])
    for _, est, mean, se in ref:
        assert abs(est - v1["expected_effective_mass_each_lag"]) <= tol
        assert abs(mean - v2["expected_jackknife_mean_each_lag"]) <= tol
        assert abs(se - v2["expected_standard_error_each_lag"]) <= tol
    got = A.cosh_effective_mass_with_jackknife(full, jk, v1["analysis_lags"])
    assert got.time_extent == 16 and got.jackknife_replicates == 5
    assert [(p.tau, p.full_estimate, p.jackknife_mean, p.standard_error) for p in got.points] == ref
    assert np.array_equal(A.analytic_periodic_single_state(16, 0.5, 1.0), np.array(full))
    v3 = vec(golden, g, "amplitude-cancellation")
    f2 = A.analytic_periodic_single_state(16, v3["full_mass"], v3["full_amplitude"])
    j2 = [A.analytic_periodic_single_state(16, m, v3["replica_amplitude"]) for m in v2["replica_masses"]]
    r2 = A.cosh_effective_mass_with_jackknife(f2, j2, [v3["analysis_lag"]])
    assert abs(r2.points[0].full_estimate - v3["expected_effective_mass"]) <= tol


def test_effective_mass_matches_oracle_on_noisy_correlators():
    rng = np.random.default_rng(0x3D)
    for nt, nrep in ((4, 3), (10, 7), (16, 12), (64, 64)):
        full = np.array(O.analytic_periodic_single_state(nt, 0.37, 2.0))
        full *= 1.0 + 0.002 * rng.standard_normal(nt)
        jk = [full * (1.0 + 0.01 * rng.standard_normal(nt)) for _ in range(nrep)]
        lags = [t for t in range(1, nt - 1) if 2 * t < nt]
        ref = O.cosh_effective_mass_with_jackknife(full, jk, lags)
        got = A.cosh_effective_mass_with_jackknife(full, jk, lags)
        assert [(p.tau, p.full_estimate, p.jackknife_mean, p.standard_error) for p in got.points] == ref


def test_effective_mass_fails_closed_like_the_reference(golden):
    full, jk = canonical_em()
    bad = full.copy()
    bad[2] = 0.0
    assert variant_of(A.cosh_effective_mass_with_jackknife, bad, jk, [2]) == "NonPositiveCentralCorrelator"
    bad = full.copy()
    bad[2] = 10.0
    assert variant_of(A.cosh_effective_mass_with_jackknife, bad, jk, [2]) == "AcoshDomainViolation"
    ragged = [r.copy() for r in jk]
    ragged[0] = ragged[0][:-1]
    assert variant_of(A.cosh_effective_mass_with_jackknife, full, ragged, [2]) == "ShapeMismatch"
    assert variant_of(A.cosh_effective_mass_with_jackknife, full, [full, full], [2]) == \
        "TooFewJackknifeReplicates"
    assert variant_of(A.cosh_effective_mass_with_jackknife, full, [full] * 65, [2]) == \
        "TooManyJackknifeReplicates"
    assert variant_of(A.cosh_effective_mass_with_jackknife, full, jk, []) == "EmptyAnalysisWindow"
    for lags in ([0], [8], [2, 2], [3, 2], [2**64 - 1]):
        assert variant_of(A.cosh_effective_mass_with_jackknife, full, jk, lags) == "InvalidAnalysisLag"
    bad = full.copy()
    bad[1] = np.nan
    assert variant_of(A.cosh_effective_mass_with_jackknife, bad, jk, [2]) == "NonFiniteCorrelator"
    jb = [r.copy() for r in jk]
    jb[0][1] = np.inf
    assert variant_of(A.cosh_effective_mass_with_jackknife, full, jb, [2]) == "NonFiniteCorrelator"
    assert variant_of(A.cosh_effective_mass_with_jackknife, full[:3], [full[:3]] * 3, [1]) == \
        "TimeExtentTooSmall"
    assert variant_of(A.analytic_periodic_single_state, 16, 0.0, 1.0) == "InvalidFixtureParameter"
    assert variant_of(A.analytic_periodic_single_state, 65, 0.5, 1.0) == "InvalidFixtureParameter"
    # the oracle fails the same way
    assert oracle_variant(O.cosh_effective_mass_with_jackknife, full, jk, [3, 2]) == "InvalidAnalysisLag"


# ------------------------------------------------------------ phase 3E

def _fit_tuple(r: A.ScalarFitResult):
    return dict(time_extent=r.time_extent, jackknife_replicates=r.jackknife_replicates,
                selected_window=(r.selected_window.start, r.selected_window.end),
                plateau_weighted_effective_mass=r.plateau_weighted_effective_mass,
                plateau_maximum_z=r.plateau_maximum_z, fitted_mass=r.fitted_mass,
                fitted_amplitude=r.fitted_amplitude, chi_square=r.chi_square,
                degrees_of_freedom=r.degrees_of_freedom, chi_square_per_dof=r.chi_square_per_dof,
                mass_jackknife_mean=r.mass_jackknife_mean, mass_standard_error=r.mass_standard_error,
                amplitude_jackknife_mean=r.amplitude_jackknife_mean,
                amplitude_standard_error=r.amplitude_standard_error,
                maximum_off_diagonal_correlation=r.maximum_off_diagonal_correlation)


def test_scalar_fit_golden_oracle_and_engine(golden):
    g = "glueball-scalar-fit-phase3e-v1.json"
    v = vec(golden, g, "canonical-correlated-single-state-fit")
    vc = vec(golden, g, "correlated-covariance-not-diagonal")
    vj = vec(golden, g, "jackknife-parameter-refit")
    tol = v["absolute_tolerance"]
    full, jk, cands = A.canonical_scalar_fit_fixture()
    assert [(w.start, w.end) for w in cands] == [tuple(w) for w in v["candidate_windows"]]
    assert np.array_equal(full, np.array(O.analytic_periodic_single_state(16, 0.5, 1.0)))
    ref = O.correlated_scalar_fit(full, jk, [(w.start, w.end) for w in cands])
    got = _fit_tuple(A.correlated_scalar_fit(full, jk, cands))
    assert got == ref
    assert list(got["selected_window"]) == v["expected_selected_window"]
    assert abs(got["plateau_weighted_effective_mass"] - v["expected_plateau_weighted_effective_mass"]) <= tol
    assert got["plateau_maximum_z"] <= 1.0e-10
    assert abs(got["fitted_mass"] - v["expected_fitted_mass"]) <= 1.0e-15
    assert abs(got["fitted_amplitude"] - v["expected_fitted_amplitude"]) <= tol
    assert abs(got["chi_square"] - v["expected_chi_square"]) <= tol
    assert got["degrees_of_freedom"] == v["expected_degrees_of_freedom"]
    assert abs(got["mass_jackknife_mean"] - vj["expected_mass_jackknife_mean"]) <= 1.0e-15
    assert abs(got["mass_standard_error"] - vj["expected_mass_standard_error"]) <= tol
    assert got["amplitude_standard_error"] > 0.0
    assert abs(got["maximum_off_diagonal_correlation"] -
               vc["expected_maximum_off_diagonal_correlation"]) <= tol
    # the replica grid masses the vector lists
    inv = O.invert_matrix(O.jackknife_covariance([list(r) for r in jk], (3, 6)))
    masses = [O.profile_grid_fit(16, (3, 6), list(r[3:7]), inv)[0] for r in jk]
    assert masses == pytest.approx(vj["replica_mass_grid_results"], abs=1e-12)


def test_scalar_fit_covariance_pieces_match_oracle():
    full, jk, _ = A.canonical_scalar_fit_fixture()
    w = A.FitWindow(3, 6)
    cov = A.jackknife_covariance(jk, w)
    ref_cov = O.jackknife_covariance([list(r) for r in jk], (3, 6))
    assert np.array_equal(cov, np.array(ref_cov))
    assert np.array_equal(A.invert_matrix(cov), np.array(O.invert_matrix(ref_cov)))
    base = A.maximum_off_diagonal_correlation(cov)
    assert base == O.maximum_off_diagonal_correlation(ref_cov)
    assert abs(base - 1.0 / 17.0) <= A.SCALAR_FIT_ANALYTIC_REPLAY_TOLERANCE
    scaled = cov * 1.0e200
    assert np.all(np.isfinite(scaled))
    assert abs(A.maximum_off_diagonal_correlation(scaled) - base) <= A.SCALAR_FIT_ANALYTIC_REPLAY_TOLERANCE


def test_scalar_fit_matches_oracle_on_seeded_replicas():
    rng = np.random.default_rng(0x3E)
    for nt, nrep, mass in ((16, 8, 0.5), (12, 6, 0.8), (20, 10, 0.31)):
        full = np.array(O.analytic_periodic_single_state(nt, mass, 1.3))
        jk = [full * (1.0 + 0.004 * rng.standard_normal(nt)) for _ in range(nrep)]
        cands = [(1, 3), (2, 5), (2, 4), (3, 5)]
        cands = [w for w in cands if 2 * w[1] < nt]
        try:
            ref = O.correlated_scalar_fit(full, jk, cands)
        except O.AnalysisError as e:
            assert variant_of(A.correlated_scalar_fit, full, jk, [A.FitWindow(*w) for w in cands]) == e.variant
            continue
        got = _fit_tuple(A.correlated_scalar_fit(full, jk, [A.FitWindow(*w) for w in cands]))
        assert got == ref


def test_scalar_fit_fails_closed_like_the_reference():
    full, jk, _ = A.canonical_scalar_fit_fixture()
    F = A.FitWindow
    assert variant_of(A.correlated_scalar_fit, full, jk, []) == "EmptyCandidateWindows"
    for c in ([F(0, 3)], [F(2, 3)], [F(3, 8)], [F(5, 4)], [F(1, 9)]):
        assert variant_of(A.correlated_scalar_fit, full, jk, c) == "InvalidCandidateWindow"
    assert variant_of(A.correlated_scalar_fit, full, jk, [F(2, 5), F(2, 5)]) == "DuplicateCandidateWindow"
    assert variant_of(A.correlated_scalar_fit, full, jk, [F(1, 3)] * 17) == "TooManyCandidateWindows"
    assert variant_of(A.correlated_scalar_fit, full, jk[:4], [F(3, 6)]) == \
        "InsufficientReplicatesForCovariance"
    same = [full.copy() for _ in range(8)]
    # identical replicas: zero jackknife error, so no window passes the plateau gate
    assert variant_of(A.correlated_scalar_fit, full, same, [F(3, 6)]) == "NoAcceptedPlateauWindow"
    cov = A.jackknife_covariance(same, F(3, 6))
    assert variant_of(A.invert_matrix, cov) == "CovarianceNotPositiveDefinite"
    assert oracle_variant(O.invert_matrix, cov.tolist()) == "CovarianceNotPositiveDefinite"
    # an effective-mass failure inside the plateau scan keeps its own variant
    bad = full.copy()
    bad[3] = 0.0
    assert variant_of(A.correlated_scalar_fit, bad, jk, [F(3, 6)]) == "NonPositiveCentralCorrelator"
    bad[3] = full[3]
    bad[4] = 0.0   # lag 3 sees the low neighbour first
    assert variant_of(A.correlated_scalar_fit, bad, jk, [F(3, 6)]) == "AcoshDomainViolation"
    assert oracle_variant(O.correlated_scalar_fit, bad, jk, [(3, 6)]) == "AcoshDomainViolation"


# ------------------------------------------------------------ phase 3J

def _proj(p: A.PrincipalProjection):
    return p.principal_eigenvalue, tuple(p.coefficients), list(p.projected_correlator)


def test_gevp_golden_oracle_and_engine(golden):
    v = vec(golden, "glueball-scalar-variational-phase3j-v1.json", "canonical-two-state-gevp")
    mats = A.canonical_two_state_matrices()
    ref = O.principal_generalized_projection(mats.tolist(), 1, 2)
    assert abs(ref[0] - v["expected_principal_eigenvalue"]) <= 2.0e-15
    got = A.principal_generalized_projection(mats)
    assert _proj(got) == (ref[0], ref[1], ref[2])
    assert got.projected_correlator[1] == v["projected_reference_value"]

    def w(m, t):
        return math.exp(-m * t) + math.exp(-m * (16 - t))
    for t in range(16):
        assert abs(got.projected_correlator[t] - w(0.4, t) / w(0.4, 1)) <= 2.0e-11


@pytest.mark.parametrize("scales", [(3.0, 0.25), (1.0e-8, 1.0), (1.0e16, 1.0)])
def test_gevp_is_invariant_under_basis_rescaling_and_permutation(scales):
    mats = A.canonical_two_state_matrices()
    base = A.principal_generalized_projection(mats)
    for m2 in ([A.matrix_scale_basis(m, scales) for m in mats], [A.matrix_swap_basis(m) for m in mats]):
        other = A.principal_generalized_projection(np.array(m2))
        assert abs(other.principal_eigenvalue - base.principal_eigenvalue) <= 2.0e-12
        assert np.max(np.abs(other.projected_correlator - base.projected_correlator)) <= 2.0e-11
        ref = O.principal_generalized_projection(np.array(m2).tolist(), 1, 2)
        assert _proj(other) == (ref[0], ref[1], ref[2])


def test_gevp_known_answers_at_extreme_ranges():
    I = [[1.0, 0.0], [0.0, 1.0]]
    cases = [
        ([I, I, [[-1.0e16, 0.0], [0.0, 1.0]]], 1.0, (0.0, 1.0), [1.0, 1.0, 1.0]),
        ([I, I, [[1.0 + 1.0e-14, 0.0], [0.0, 1.0]]], 1.0 + 1.0e-14, (1.0, 0.0), [1.0, 1.0, 1.0 + 1.0e-14]),
        ([I, I, [[-1.0e308, 0.0], [0.0, 1.0e-308]]], 1.0e-308, (0.0, 1.0), [1.0, 1.0, 1.0e-308]),
    ]
    for mats, lam, coef, proj in cases:
        got = A.principal_generalized_projection(np.array(mats))
        assert got.principal_eigenvalue == lam and got.coefficients == coef
        assert list(got.projected_correlator) == proj
        assert O.principal_generalized_projection(mats, 1, 2) == (lam, coef, proj)
    for tiny in (MIN_SUBNORMAL, 1.0e-308, 1.0e-100, 1.0e-10):
        mats = [[[-FMAX, 0.0], [0.0, tiny]], I, [[-FMAX, 0.0], [0.0, tiny]], [[-FMAX, 0.0], [0.0, -tiny]]]
        for scales in ((1.0, 1.0), (0.5, 2.0), (-0.5, -2.0)):
            for swap in (False, True):
                inp = [A.matrix_scale_basis(m, scales) for m in mats]
                if swap:
                    inp = [A.matrix_swap_basis(m) for m in inp]
                got = A.principal_generalized_projection(np.array(inp))
                assert got.principal_eigenvalue == tiny
                assert list(got.projected_correlator) == [tiny, 1.0, tiny, -tiny]
    # tiny off-diagonal keeps a unique direction
    got = A.principal_generalized_projection(np.array([I, I, [[1.0, 1.0e-16], [1.0e-16, 1.0]]]))
    assert abs(got.coefficients[0] - math.sqrt(0.5)) <= 2.0e-15
    assert abs(got.coefficients[1] - math.sqrt(0.5)) <= 2.0e-15
    # repeated ill-conditioned reference lags project to the same bits
    e = 2.0e-14
    c0 = [[1.0, 1.0 - e], [1.0 - e, 1.0]]
    c1 = [[1.0 + e / 2.0, 1.0 - 3.0 * e / 2.0], [1.0 - 3.0 * e / 2.0, 1.0 + e / 2.0]]
    got = A.principal_generalized_projection(np.array([c0, c0, c1]))
    assert got.projected_correlator[0] == got.projected_correlator[1]
    assert abs(got.projected_correlator[0] - 1.0) <= A.NORMALIZATION_TOLERANCE
    # ill-conditioned but positive-definite reference
    got = A.principal_generalized_projection(np.array([[[1.0, 0.999999], [0.999999, 1.0]]] * 2 +
                                                      [[[2.0, 0.3], [0.3, 1.0]]]))
    assert got.principal_eigenvalue > 0.0
    assert abs(got.projected_correlator[1] - 1.0) <= A.NORMALIZATION_TOLERANCE


def test_gevp_matches_oracle_on_seeded_two_state_series():
    rng = np.random.default_rng(0x3A)
    for _ in range(40):
        nt = int(rng.integers(3, 20))
        m0, m1 = sorted(rng.uniform(0.1, 1.5, 2))
        a0, a1 = rng.uniform(0.2, 2.0, 2)
        g, x = rng.uniform(-1, 1, 2), rng.uniform(-1, 1, 2)
        mats = []
        for t in range(nt):
            w0 = a0 * (math.exp(-m0 * t) + math.exp(-m0 * (nt - t)))
            w1 = a1 * (math.exp(-m1 * t) + math.exp(-m1 * (nt - t)))
            mats.append([[w0 * g[r] * g[c] + w1 * x[r] * x[c] for c in range(2)] for r in range(2)])
        mats = (np.array(mats) * rng.uniform(1e-3, 1e3)).tolist()
        try:
            ref = O.principal_generalized_projection(mats, 1, 2)
        except O.AnalysisError as e:
            assert variant_of(A.principal_generalized_projection, np.array(mats)) == e.variant
            continue
        assert _proj(A.principal_generalized_projection(np.array(mats))) == ref


def test_gevp_fails_closed_like_the_reference():
    I = [[1.0, 0.0], [0.0, 1.0]]
    P = A.principal_generalized_projection
    assert variant_of(P, np.array([I, I, I])) == "DegeneratePrincipalEigenvector"
    assert variant_of(P, np.array([[[1.0, 0.5], [0.5, 1.0]]] * 2 + [[[-1.0e10, 0.0], [0.0, -1.0e-10]]])) == \
        "NonPositivePrincipalEigenvalue"
    c0 = [[1.0, 1.0 - 1.0e-13], [1.0 + 1.0e-13, 1.0]]
    assert variant_of(P, np.array([c0, c0, I])) == "ReferenceMatrixNotPositiveDefinite"
    mats = A.canonical_two_state_matrices()
    m = mats.copy()
    m[1] = [[1.0, 1.0], [1.0, 1.0]]
    assert variant_of(P, m) == "ReferenceMatrixNotPositiveDefinite"
    m = mats.copy()
    m[3][0][1] += 1.0e-6
    assert variant_of(P, m) == "MatrixNotSymmetric"
    assert variant_of(P, mats, 2, 2) == "InvalidReferenceTimes"
    assert variant_of(P, mats, 0, 1) == "InvalidReferenceTimes"
    m = mats.copy()
    m[0][0][0] = np.nan
    assert variant_of(P, m) == "NonFiniteAccumulator"
    assert variant_of(P, mats[:2]) == "CorrelatorShapeMismatch"
    first = np.array([[[FMAX, 0.0], [0.0, 1.0]]] * 3)
    assert variant_of(A.max_matrix_series_residual, first, -first) == "NonFiniteAccumulator"


def test_variational_correlator_from_samples_matches_oracle():
    rng = np.random.default_rng(0x3F)
    for ncfg, nt in ((1, 3), (5, 8), (16, 12)):
        p = 0.6 + 0.05 * rng.standard_normal((ncfg, nt))
        r = 0.4 + 0.05 * rng.standard_normal((ncfg, nt))
        got = A.variational_correlator_from_samples(p, r)
        (v0, v1), mats = O.variational_correlator_from_samples(p.tolist(), r.tolist())
        assert got.vacuum_means == (v0, v1)
        assert np.array_equal(got.matrices, np.array(mats))
        assert all(m[0][1] == m[1][0] for m in got.matrices)
    assert variant_of(A.variational_correlator_from_samples, np.zeros((65, 4)), np.zeros((65, 4))) == \
        "TooManyConfigurations"
    assert variant_of(A.variational_correlator_from_samples, np.zeros((2, 2)), np.zeros((2, 2))) == \
        "TimeExtentTooSmall"
    bad = np.ones((2, 4))
    bad[1, 2] = np.inf
    assert variant_of(A.variational_correlator_from_samples, bad, np.ones((2, 4))) == "NonFiniteObservable"
