"""Host analysis of glueball correlators -- mirror of the reference modules
``glueball_effective_mass`` (phase 3D), ``glueball_scalar_fit`` (phase 3E)
and ``glueball_scalar_variational`` (phase 3J).

The arithmetic is libymgpu's host FP64 (``include/ym_analysis.h``); the
operator samples the variational correlator consumes come from the device
(``Ensemble.scalar_operator_basis``).  Names, argument meaning and error
variants follow the reference, so callers and tests read like the
reference's own.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import _lib as L
from ._lib import lib
from .errors import VARIANTS, YmError, check

# glueball_effective_mass.rs:16-22
EFFECTIVE_MASS_CONTRACT_ID = "YM-GLUEBALL-EFFECTIVE-MASS-V1"
EFFECTIVE_MASS_STATUS = "phase-3d-frozen"
MIN_JACKKNIFE_REPLICATES = 3
MAX_JACKKNIFE_REPLICATES = 64
MIN_TIME_EXTENT = 4
MAX_TIME_EXTENT = 64
EFFECTIVE_MASS_ANALYTIC_REPLAY_TOLERANCE = 2.0e-12
# glueball_scalar_fit.rs:13-26
SCALAR_FIT_CONTRACT_ID = "YM-GLUEBALL-SCALAR-FIT-V1"
SCALAR_FIT_STATUS = "phase-3e-frozen"
MIN_WINDOW_POINTS = 3
MAX_WINDOW_POINTS = 8
MAX_CANDIDATE_WINDOWS = 16
PLATEAU_MAX_Z = 2.5
MASS_GRID_MIN = 0.05
MASS_GRID_MAX = 2.0
MASS_GRID_STEP = 0.001
MASS_GRID_STEPS = 1950
COVARIANCE_PIVOT_REL_TOLERANCE = 1.0e-12
SCALAR_FIT_ANALYTIC_REPLAY_TOLERANCE = 2.0e-10
CANONICAL_PERTURBATION = 0.005
CANONICAL_SHARED_CORRELATION = 0.25
# glueball_scalar_variational.rs:21-37
VARIATIONAL_CONTRACT_ID = "YM-GLUEBALL-SCALAR-VARIATIONAL-BASIS-V1"
VARIATIONAL_STATUS = "phase-3j-candidate"
BASIS_DIMENSION = 2
REFERENCE_TIME = 1
DIAGONALIZATION_TIME = 2
SYMMETRY_TOLERANCE = 2.0e-12
GAUGE_INVARIANCE_TOLERANCE = 5.0e-11
NORMALIZATION_TOLERANCE = 2.0e-12
POSITIVE_DEFINITE_PIVOT_TOLERANCE = 1.0e-14
CANONICAL_TIME_EXTENT = 16
CANONICAL_GROUND_MASS = 0.4
CANONICAL_EXCITED_MASS = 0.9
CANONICAL_GROUND_AMPLITUDE = 1.2
CANONICAL_EXCITED_AMPLITUDE = 0.8
CANONICAL_GROUND_COUPLING = (1.0, 0.5)
CANONICAL_EXCITED_COUPLING = (0.25, 1.0)
GOLDEN_CANONICAL_PRINCIPAL_EIGENVALUE = 0.673346666250657


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _p(a: np.ndarray):
    return a.ctypes.data_as(L.P(L.f64))


class _Replicas:
    """A jackknife set as the reference's &[Vec<f64>] (ragged allowed)."""

    def __init__(self, jackknife: Sequence[Sequence[float]]):
        self.rows = [_f64(r) for r in jackknife]
        n = len(self.rows)
        self.ptrs = (L.P(L.f64) * max(n, 1))(*[_p(r) for r in self.rows])
        self.lens = (L.i64 * max(n, 1))(*[r.size for r in self.rows])
        self.n = n


# ------------------------------------------------------------ phase 3D

@dataclass(frozen=True)
class EffectiveMassPoint:
    tau: int
    full_estimate: float
    jackknife_mean: float
    standard_error: float


@dataclass(frozen=True)
class EffectiveMassSeries:
    time_extent: int
    jackknife_replicates: int
    points: List[EffectiveMassPoint]


def cosh_effective_mass_with_jackknife(full, jackknife, lags) -> EffectiveMassSeries:
    """glueball_effective_mass.rs:170-234: m_eff(tau) = acosh((C(tau-1) +
    C(tau+1)) / (2 C(tau))) on the lags, with the delete-one jackknife error
    sqrt((N-1)/N sum_i (m_i - m_bar)^2)."""
    f = _f64(full)
    jk = _Replicas(jackknife)
    lag_arr = (L.u64 * max(len(lags), 1))(*[int(t) for t in lags])
    pts = (L.EffectiveMassPoint * max(len(lags), 1))()
    check(lib().ym_cosh_effective_mass_with_jackknife(_p(f), f.size, jk.ptrs, jk.lens, jk.n, lag_arr,
                                                      len(lags), pts),
          "cosh_effective_mass_with_jackknife")
    return EffectiveMassSeries(f.size, jk.n, [
        EffectiveMassPoint(p.tau, p.full_estimate, p.jackknife_mean, p.standard_error)
        for p in pts[:len(lags)]])


def analytic_periodic_single_state(time_extent: int, mass: float, amplitude: float) -> np.ndarray:
    """glueball_effective_mass.rs:237-263: A (exp(-m tau) + exp(-m (N_t - tau)))."""
    out = np.zeros(max(int(time_extent), 1))
    check(lib().ym_analytic_periodic_single_state(int(time_extent), float(mass), float(amplitude),
                                                  _p(out)), "analytic_periodic_single_state")
    return out[:time_extent]


# ------------------------------------------------------------ phase 3E

@dataclass(frozen=True)
class FitWindow:
    start: int
    end: int

    def point_count(self):
        return self.end - self.start + 1 if self.end >= self.start else None

    def _c(self) -> L.FitWindowC:
        return L.FitWindowC(self.start, self.end)


@dataclass(frozen=True)
class ScalarFitResult:
    time_extent: int
    jackknife_replicates: int
    selected_window: FitWindow
    plateau_weighted_effective_mass: float
    plateau_maximum_z: float
    fitted_mass: float
    fitted_amplitude: float
    chi_square: float
    degrees_of_freedom: int
    chi_square_per_dof: float
    mass_jackknife_mean: float
    mass_standard_error: float
    amplitude_jackknife_mean: float
    amplitude_standard_error: float
    maximum_off_diagonal_correlation: float


def correlated_scalar_fit(full, jackknife, candidate_windows: Sequence[FitWindow]) -> ScalarFitResult:
    """glueball_scalar_fit.rs:595-650: plateau window (longest passing, ties to
    the later start), full jackknife covariance, profile-grid correlated
    single-state fit of the full correlator and of every replica."""
    f = _f64(full)
    jk = _Replicas(jackknife)
    n = len(candidate_windows)
    wins = (L.FitWindowC * max(n, 1))(*[w._c() for w in candidate_windows])
    r = L.ScalarFitResultC()
    check(lib().ym_correlated_scalar_fit(_p(f), f.size, jk.ptrs, jk.lens, jk.n, wins, n, C.byref(r)),
          "correlated_scalar_fit")
    return ScalarFitResult(
        r.time_extent, r.jackknife_replicates,
        FitWindow(r.selected_window.start, r.selected_window.end),
        r.plateau_weighted_effective_mass, r.plateau_maximum_z, r.fitted_mass, r.fitted_amplitude,
        r.chi_square, r.degrees_of_freedom, r.chi_square_per_dof, r.mass_jackknife_mean,
        r.mass_standard_error, r.amplitude_jackknife_mean, r.amplitude_standard_error,
        r.maximum_off_diagonal_correlation)


def jackknife_covariance(jackknife, window: FitWindow) -> np.ndarray:
    """glueball_scalar_fit.rs:276-322 over ragged replicas."""
    jk = _Replicas(jackknife)
    pc = window.point_count() or 0
    out = np.zeros((max(pc, 1), max(pc, 1)))
    check(lib().ym_scalar_fit_window_covariance(jk.ptrs, jk.lens, jk.n, window._c(), _p(out)),
          "jackknife_covariance")
    return out[:pc, :pc]


def invert_matrix(matrix) -> np.ndarray:
    """glueball_scalar_fit.rs:361-421 (positive-definite check, then
    Gauss-Jordan with partial pivoting)."""
    m = _f64(matrix)
    n = m.shape[0] if m.ndim == 2 else 0
    out = np.zeros((max(n, 1), max(n, 1)))
    check(lib().ym_scalar_fit_invert_covariance(_p(m), n, _p(out)), "invert_matrix")
    return out[:n, :n]


def maximum_off_diagonal_correlation(covariance) -> float:
    """glueball_scalar_fit.rs:567-593."""
    m = _f64(covariance)
    out = L.f64()
    check(lib().ym_maximum_off_diagonal_correlation(_p(m), m.shape[0], C.byref(out)),
          "maximum_off_diagonal_correlation")
    return out.value


def canonical_scalar_fit_fixture() -> Tuple[np.ndarray, List[np.ndarray], List[FitWindow]]:
    """glueball_scalar_fit.rs:663-690."""
    full = np.zeros(16)
    jk = np.zeros((8, 16))
    wins = (L.FitWindowC * 3)()
    check(lib().ym_canonical_scalar_fit_fixture(_p(full), _p(jk), wins), "canonical_scalar_fit_fixture")
    return full, [row.copy() for row in jk], [FitWindow(w.start, w.end) for w in wins]


# ------------------------------------------------------------ phase 3J

@dataclass(frozen=True)
class ScalarVariationalCorrelator:
    configuration_count: int
    time_extent: int
    vacuum_means: Tuple[float, float]
    matrices: np.ndarray   # [time][2][2]


@dataclass(frozen=True)
class PrincipalProjection:
    reference_time: int
    diagonalization_time: int
    principal_eigenvalue: float
    coefficients: Tuple[float, float]
    projected_correlator: np.ndarray


def variational_correlator_from_samples(plaquette, rectangle) -> ScalarVariationalCorrelator:
    """The symmetric connected cross-correlator of
    glueball_scalar_variational.rs:628-744 from operator samples
    plaquette[cfg][t], rectangle[cfg][t]."""
    p, r = _f64(plaquette), _f64(rectangle)
    if p.ndim != 2 or p.shape != r.shape:
        raise YmError(VARIANTS["CorrelatorShapeMismatch"], "scalar_variational_connected_correlator")
    ncfg, nt = p.shape
    samples = np.ascontiguousarray(np.stack([p, r], axis=-1))
    means = np.zeros(2)
    mats = np.zeros((max(nt, 1), 2, 2))
    check(lib().ym_scalar_variational_connected_correlator(_p(samples), ncfg, nt, _p(means), _p(mats)),
          "scalar_variational_connected_correlator")
    return ScalarVariationalCorrelator(ncfg, nt, (means[0], means[1]), mats[:nt])


def scalar_variational_connected_correlator(ens) -> ScalarVariationalCorrelator:
    """glueball_scalar_variational.rs:628-744 with the chains of an SU(3)
    ``Ensemble`` as the configurations: the operator basis runs on the
    device, the correlator matrix on the host."""
    from .glueball import operator_samples
    if ens.n_chains == 0:
        raise YmError(VARIANTS["EmptyConfigurationSet"], "scalar_variational_connected_correlator")
    if any(e != ens.extents[0] for e in ens.extents):
        raise YmError(VARIANTS["LatticeExtentsMismatch"], "scalar_variational_connected_correlator")
    p, r = operator_samples(ens)
    return variational_correlator_from_samples(p, r)


def principal_generalized_projection(matrices, reference_time: int = REFERENCE_TIME,
                                     diagonalization_time: int = DIAGONALIZATION_TIME
                                     ) -> PrincipalProjection:
    """glueball_scalar_variational.rs:746-925: largest generalized eigenvalue of
    C(t1) v = lambda C(t0) v by Cholesky whitening of C(t0), v normalised to
    v^T C(t0) v = 1, and the projected correlator v^T C(t) v."""
    m = _f64(matrices)
    nt = m.shape[0] if m.ndim == 3 else 0
    if m.ndim != 3 or m.shape[1:] != (2, 2):
        raise YmError(VARIANTS["CorrelatorShapeMismatch"], "principal_generalized_projection")
    res = L.PrincipalProjectionC()
    proj = np.zeros(max(nt, 1))
    check(lib().ym_principal_generalized_projection(_p(m), nt, int(reference_time),
                                                    int(diagonalization_time), C.byref(res), _p(proj)),
          "principal_generalized_projection")
    return PrincipalProjection(res.reference_time, res.diagonalization_time, res.principal_eigenvalue,
                               (res.coefficients[0], res.coefficients[1]), proj[:nt])


def canonical_two_state_matrices() -> np.ndarray:
    """glueball_scalar_variational.rs:931-951: [16][2][2]."""
    out = np.zeros((CANONICAL_TIME_EXTENT, 2, 2))
    check(lib().ym_canonical_two_state_matrices(_p(out)), "canonical_two_state_matrices")
    return out


def max_matrix_series_residual(first, second) -> float:
    """glueball_scalar_variational.rs:953-975."""
    a, b = _f64(first), _f64(second)
    out = L.f64()
    check(lib().ym_max_matrix_series_residual(_p(a), a.shape[0], _p(b), b.shape[0], C.byref(out)),
          "max_matrix_series_residual")
    return out.value


def matrix_scale_basis(matrix, scales) -> np.ndarray:
    """glueball_scalar_variational.rs:605-616 (test helper)."""
    m = _f64(matrix)
    s0, s1 = scales
    return np.array([[s0 * m[0, 0] * s0, s0 * m[0, 1] * s1], [s1 * m[1, 0] * s0, s1 * m[1, 1] * s1]])


def matrix_swap_basis(matrix) -> np.ndarray:
    """glueball_scalar_variational.rs:618-620 (test helper)."""
    m = _f64(matrix)
    return np.array([[m[1, 1], m[1, 0]], [m[0, 1], m[0, 0]]])
