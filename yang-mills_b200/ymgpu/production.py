"""The phase-3F scalar glueball production campaign -- mirror of the reference
module ``glueball_scalar_production`` (run_production_scalar_analysis,
glueball_scalar_production.rs:640-720).

Sixteen independent 4^3x10 chains at beta 5.7 run their 64 + 4 Metropolis
sweeps in one device ensemble; raw, one-level and two-level stout
transforms, the A1++ operator samples and the correlators come from the
device and the host analysis (the connected correlator and its replay
check, delete-one jackknife, the correlated single-state fit per surface,
window / operator / transformation stability).  Failures of the fit that
the reference records as scientific outcomes become surface error codes;
the others propagate, as in the reference.

The chains are the engine's (checkerboard order, counter-based streams), so
they are different configurations from the reference's run; every rule the
summary applies is the reference's.
"""
from __future__ import annotations

import ctypes
import ctypes.util
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from . import analysis as A
from . import glueball as G
from .errors import VARIANTS, YmError

PRODUCTION_CONTRACT_ID = "YM-GLUEBALL-SCALAR-PRODUCTION-V1"
PRODUCTION_STATUS = "phase-3f-frozen"
EXTENTS = (4, 4, 4, 10)
BETA = 5.7
MASTER_SEED = 0x3F00_2026_0915_0001
CHAIN_COUNT = 16
THERMALIZATION_SWEEPS = 64
POST_THERMALIZATION_SWEEPS = 4
TOTAL_SWEEPS_PER_CHAIN = THERMALIZATION_SWEEPS + POST_THERMALIZATION_SWEEPS
PROPOSAL_ANGLE = 0.35
LINKS_PER_SWEEP = 4 * 4 * 4 * 10 * 4
PROPOSALS_PER_LINK = 8
EXPECTED_PROPOSALS_PER_CHAIN = LINKS_PER_SWEEP * PROPOSALS_PER_LINK * TOTAL_SWEEPS_PER_CHAIN
MIN_ACCEPTANCE = 0.10
MAX_ACCEPTANCE = 0.95
STOUT_LEVELS = (1, 2)
TRANSFORMATION_LABELS = ("raw", "stout-1", "stout-2")
PRIMARY_TRANSFORMATION = "stout-2"
PRIMARY_OPERATOR = "plaquette-1x1"
OPERATORS = ("plaquette-1x1", "rectangle-2x1")
STABILITY_MAX_Z = 5.0
CORRELATOR_REPLAY_TOLERANCE = 2.0e-12
CANDIDATE_WINDOWS = (A.FitWindow(1, 3), A.FitWindow(2, 4), A.FitWindow(1, 4))
OBSERVED_REJECTION_CODE = "effective-mass-rejected"
OBSERVED_SURFACE_OUTCOMES = tuple((t, o, OBSERVED_REJECTION_CODE)
                                  for t in TRANSFORMATION_LABELS for o in OPERATORS)
LINK_RESIDUAL_LIMIT = 5.0e-12

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.hypot.argtypes = [ctypes.c_double, ctypes.c_double]
_libm.hypot.restype = ctypes.c_double


@dataclass(frozen=True)
class ChainEvidence:
    chain_id: int
    derived_seed: int
    proposals: int
    accepts: int
    acceptance: float
    plaquette: float
    unitarity_residual: float
    determinant_residual: float


@dataclass
class CorrelatorEvidence:
    full: np.ndarray
    jackknife: List[np.ndarray]


@dataclass
class SurfaceOutcome:
    transformation: str
    operator: str
    fit: Optional[A.ScalarFitResult]
    error_code: Optional[str]

    def succeeded(self) -> bool:
        return self.fit is not None


@dataclass
class SurfaceRecord:
    outcome: SurfaceOutcome
    correlator: CorrelatorEvidence


@dataclass
class ProductionSummary:
    chain_evidence: List[ChainEvidence] = field(default_factory=list)
    surfaces: List[SurfaceRecord] = field(default_factory=list)
    sampler_diagnostics_passed: bool = False
    primary_window_successes: int = 0
    primary_window_max_z: Optional[float] = None
    operator_stability_z: Optional[float] = None
    transformation_stability_successes: int = 0
    transformation_stability_max_z: Optional[float] = None
    scalar_pipeline_validated: bool = False


_SCIENTIFIC = {   # scientific_fit_error_code (glueball_scalar_production.rs:474-487)
    "DegeneratePlateauUncertainty": "degenerate-plateau-uncertainty",
    "NoAcceptedPlateauWindow": "no-accepted-plateau-window",
    "CovarianceNotPositiveDefinite": "covariance-not-positive-definite",
    "SingularCovariance": "singular-covariance",
    "NoFiniteGridFit": "no-finite-grid-fit",
    "NonPositiveCentralCorrelator": OBSERVED_REJECTION_CODE,
    "AcoshDomainViolation": OBSERVED_REJECTION_CODE,
}


def scientific_fit_error_code(variant: str) -> Optional[str]:
    return _SCIENTIFIC.get(variant)


def production_fit_error(err: YmError) -> YmError:
    """production_fit_error (glueball_scalar_production.rs:489-501)."""
    if err.variant == "AllocationFailed":
        return YmError(VARIANTS["AllocationFailed"], "production fit")
    if err.variant in ("NonFiniteStatistic", "NonFiniteCorrelator"):
        return YmError(VARIANTS["NonFiniteStatistic"], "production fit")
    return err


def stable_z(first: A.ScalarFitResult, second: A.ScalarFitResult) -> Optional[float]:
    """glueball_scalar_production.rs:550-557."""
    scale = _libm.hypot(first.mass_standard_error, second.mass_standard_error)
    if not np.isfinite(scale) or scale <= 0.0:
        return None
    z = abs(first.fitted_mass - second.fitted_mass) / scale
    return z if np.isfinite(z) else None


def maximum_pairwise_z(fits) -> Tuple[int, Optional[float]]:
    """glueball_scalar_production.rs:559-573."""
    if len(fits) < 2:
        return len(fits), None
    mx = 0.0
    for i in range(len(fits)):
        for j in range(i + 1, len(fits)):
            z = stable_z(fits[i], fits[j])
            if z is None:
                return len(fits), None
            mx = max(mx, z)
    return len(fits), mx


def _fit(correlator: CorrelatorEvidence, windows):
    try:
        return A.correlated_scalar_fit(correlator.full, correlator.jackknife, windows), None
    except YmError as e:
        code = scientific_fit_error_code(e.variant)
        if code is None:
            raise production_fit_error(e) from None
        return None, code


def analyze_surface(transformation: str, operator: str, correlator: CorrelatorEvidence) -> SurfaceRecord:
    """glueball_scalar_production.rs:503-528."""
    fit, code = _fit(correlator, CANDIDATE_WINDOWS)
    return SurfaceRecord(SurfaceOutcome(transformation, operator, fit, code), correlator)


def window_stability(primary: SurfaceRecord) -> Tuple[int, Optional[float]]:
    """glueball_scalar_production.rs:575-605: every candidate window alone."""
    fits = []
    for w in CANDIDATE_WINDOWS:
        fit, _ = _fit(primary.correlator, [w])
        if fit is not None:
            fits.append(fit)
    return maximum_pairwise_z(fits)


def correlator_evidence(samples: np.ndarray) -> CorrelatorEvidence:
    """glueball_scalar_production.rs:445-472: connected correlator of the
    samples, its replay against the frozen estimator, jackknife replicas."""
    full = G.connected_from_samples(samples)
    _, _, frozen = G.periodic_connected_estimator(samples)
    if frozen.shape != full.shape or np.any(np.abs(frozen - full) > CORRELATOR_REPLAY_TOLERANCE):
        raise YmError(VARIANTS["CorrelatorReplayMismatch"], "correlator_evidence")
    jk = G.jackknife_replicas(samples)
    return CorrelatorEvidence(full, [row.copy() for row in jk])


def summarize_surfaces(chain_evidence: List[ChainEvidence], surfaces: List[SurfaceRecord]) -> ProductionSummary:
    """The stability gates of run_production_scalar_analysis
    (glueball_scalar_production.rs:663-720) over analysed surfaces."""
    def find(t, o):
        for s in surfaces:
            if s.outcome.transformation == t and s.outcome.operator == o:
                return s
        return None

    sampler_ok = all(MIN_ACCEPTANCE <= e.acceptance <= MAX_ACCEPTANCE for e in chain_evidence)
    primary = find(PRIMARY_TRANSFORMATION, PRIMARY_OPERATOR)
    if primary is None:
        raise YmError(VARIANTS["ConfigurationShapeMismatch"], "run_production_scalar_analysis")
    pw_n, pw_z = window_stability(primary)
    a = find(PRIMARY_TRANSFORMATION, "plaquette-1x1")
    b = find(PRIMARY_TRANSFORMATION, "rectangle-2x1")
    op_z = stable_z(a.outcome.fit, b.outcome.fit) if (a and b and a.outcome.fit and b.outcome.fit) else None
    tfits = [s.outcome.fit for t in TRANSFORMATION_LABELS
             for s in [find(t, PRIMARY_OPERATOR)] if s is not None and s.outcome.fit is not None]
    t_n, t_z = maximum_pairwise_z(tfits)
    validated = (sampler_ok and primary.outcome.succeeded() and pw_n >= 2
                 and pw_z is not None and pw_z <= STABILITY_MAX_Z
                 and op_z is not None and op_z <= STABILITY_MAX_Z
                 and t_n >= 2 and t_z is not None and t_z <= STABILITY_MAX_Z)
    return ProductionSummary(chain_evidence, surfaces, sampler_ok, pw_n, pw_z, op_z, t_n, t_z, validated)


def observed_phase3f_receipt_matches(summary: ProductionSummary) -> bool:
    """glueball_scalar_production.rs:616-638."""
    surfaces_match = len(summary.surfaces) == len(OBSERVED_SURFACE_OUTCOMES) and all(
        r.outcome.transformation == t and r.outcome.operator == o and r.outcome.fit is None
        and r.outcome.error_code == code
        for r, (t, o, code) in zip(summary.surfaces, OBSERVED_SURFACE_OUTCOMES))
    return (summary.sampler_diagnostics_passed and surfaces_match
            and summary.primary_window_successes == 0 and summary.primary_window_max_z is None
            and summary.operator_stability_z is None
            and summary.transformation_stability_successes == 0
            and summary.transformation_stability_max_z is None
            and not summary.scalar_pipeline_validated)


def run_production_scalar_analysis(device: int = 0, generator_mode: str = "ordered") -> ProductionSummary:
    """The frozen phase-3F campaign with its chains on the device."""
    from .ensemble import Ensemble
    from .su3_ensemble import derive_su3_chain_seed
    seeds = [derive_su3_chain_seed(MASTER_SEED, k) for k in range(CHAIN_COUNT)]
    with Ensemble([list(EXTENTS)] * CHAIN_COUNT, BETA, seeds, device=device) as raw:
        raw.metropolis_sweeps(PROPOSAL_ANGLE, TOTAL_SWEEPS_PER_CHAIN, generator_mode)
        prop, acc = raw.accounting()
        plaq = raw.average_plaquette()
        ures, dres = raw.max_residuals()
        evidence = []
        for k in range(CHAIN_COUNT):
            if int(prop[k]) != EXPECTED_PROPOSALS_PER_CHAIN:
                raise YmError(VARIANTS["AccountingOverflow"], "run_production_scalar_analysis")
            e = ChainEvidence(k, seeds[k], int(prop[k]), int(acc[k]), float(acc[k]) / float(prop[k]),
                              float(plaq[k]), float(ures[k]), float(dres[k]))
            if not all(np.isfinite([e.acceptance, e.plaquette, e.unitarity_residual, e.determinant_residual])):
                raise YmError(VARIANTS["NonFiniteStatistic"], "run_production_scalar_analysis")
            if e.unitarity_residual > LINK_RESIDUAL_LIMIT or e.determinant_residual > LINK_RESIDUAL_LIMIT:
                raise YmError(VARIANTS["LinkResidualExceeded"], "run_production_scalar_analysis")
            evidence.append(e)
        surfaces = []
        for label, levels in zip(TRANSFORMATION_LABELS, (0,) + STOUT_LEVELS):
            ens = G.spatial_stout_smear(raw, G.CANONICAL_RHO, levels) if levels else raw
            try:
                p, r = G.operator_samples(ens)
            finally:
                if levels:
                    ens.close()
            cp, cr = correlator_evidence(p), correlator_evidence(r)
            surfaces.append(analyze_surface(label, "plaquette-1x1", cp))
            surfaces.append(analyze_surface(label, "rectangle-2x1", cr))
    return summarize_surfaces(evidence, surfaces)
