"""The scalar glueball production campaigns -- mirror of the reference modules
``glueball_scalar_production`` (phase 3F, run_production_scalar_analysis,
glueball_scalar_production.rs:640-720), ``glueball_scalar_recovery``
(phase 3G, :419), ``glueball_scalar_geometry_recovery`` (phase 3H, :491) and
``glueball_scalar_temporal_recovery`` (phase 3I, :491), with their receipt
rules (``*_receipt.rs``).

Every campaign's independent chains run their 64 + 4 Metropolis sweeps in
one device ensemble; the stout transforms, the stride-2 blocking, the A1++
operator samples and the correlators come from the device, and the host
does the analysis (connected correlator and its replay check, delete-one
jackknife, the correlated single-state fit per surface, window / operator /
transformation stability).  Failures of the fit that the reference records
as scientific outcomes become surface error codes; the others propagate, as
in the reference.

The chains are the engine's (checkerboard order, counter-based streams), so
they are different configurations from the reference's runs; every rule the
summaries apply is the reference's.
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


@dataclass(frozen=True)
class Campaign:
    """One frozen campaign: schedule, transformations and its receipt rule."""
    name: str
    contract_id: str
    extents: Tuple[int, int, int, int]
    master_seed: int
    chain_count: int
    transformations: Tuple[Tuple[str, str, int], ...]   # (label, "stout" | "block" | "raw", levels)
    primary_transformation: str
    exact_acceptance_check: bool          # acceptance == accepts / proposals bit for bit
    observed_outcomes: Optional[Tuple[Tuple[str, str, str], ...]]   # None: no recorded receipt
    check_chain_identity: bool = False    # the receipt also pins seeds and accounting

    @property
    def expected_proposals_per_chain(self) -> int:
        e = self.extents
        return e[0] * e[1] * e[2] * e[3] * 4 * PROPOSALS_PER_LINK * TOTAL_SWEEPS_PER_CHAIN


_STOUT_SCAN = (("raw", "raw", 0), ("stout-1", "stout", 1), ("stout-2", "stout", 2))
_BLOCK_SCAN = _STOUT_SCAN + (("block-1", "block", 1),)


def _rejected(scan):
    return tuple((t, o, OBSERVED_REJECTION_CODE) for t, _, _ in scan for o in OPERATORS)


CAMPAIGNS = {
    # glueball_scalar_production.rs:17-90
    "phase3f": Campaign("phase3f", "YM-GLUEBALL-SCALAR-PRODUCTION-V1", (4, 4, 4, 10),
                        0x3F00_2026_0915_0001, 16, _STOUT_SCAN, "stout-2", False, _rejected(_STOUT_SCAN)),
    # glueball_scalar_recovery.rs:34-47, glueball_scalar_recovery_receipt.rs
    "phase3g": Campaign("phase3g", "YM-GLUEBALL-SCALAR-RECOVERY-V1", (4, 4, 4, 10),
                        0x3F01_2026_0915_0001, 32, _STOUT_SCAN, "stout-2", False, _rejected(_STOUT_SCAN),
                        True),
    # glueball_scalar_geometry_recovery.rs:43-62, glueball_scalar_geometry_recovery_receipt.rs
    "phase3h": Campaign("phase3h", "YM-GLUEBALL-SCALAR-GEOMETRY-RECOVERY-V1", (6, 6, 6, 10),
                        0x3F02_2026_0915_0001, 32, _BLOCK_SCAN, "block-1", True, _rejected(_BLOCK_SCAN),
                        True),
    # glueball_scalar_temporal_recovery.rs:43-62 (a candidate: no receipt recorded)
    "phase3i": Campaign("phase3i", "YM-GLUEBALL-SCALAR-TEMPORAL-RECOVERY-V1", (6, 6, 6, 16),
                        0x3F03_2026_0927_0001, 32, _BLOCK_SCAN, "block-1", True, None),
}


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


def summarize_surfaces(chain_evidence: List[ChainEvidence], surfaces: List[SurfaceRecord],
                       campaign: "Campaign" = None) -> ProductionSummary:
    """The stability gates of run_production_scalar_analysis
    (glueball_scalar_production.rs:663-720; the recovery campaigns apply the
    same gates to their own primary surface) over analysed surfaces."""
    campaign = campaign or CAMPAIGNS["phase3f"]
    primary_t = campaign.primary_transformation
    labels = tuple(t for t, _, _ in campaign.transformations)
    def find(t, o):
        for s in surfaces:
            if s.outcome.transformation == t and s.outcome.operator == o:
                return s
        return None

    sampler_ok = all(MIN_ACCEPTANCE <= e.acceptance <= MAX_ACCEPTANCE and
                     (not campaign.exact_acceptance_check or
                      e.acceptance == float(e.accepts) / float(e.proposals)) for e in chain_evidence)
    primary = find(primary_t, PRIMARY_OPERATOR)
    if primary is None:
        raise YmError(VARIANTS["ConfigurationShapeMismatch"], "run_production_scalar_analysis")
    pw_n, pw_z = window_stability(primary)
    a = find(primary_t, "plaquette-1x1")
    b = find(primary_t, "rectangle-2x1")
    op_z = stable_z(a.outcome.fit, b.outcome.fit) if (a and b and a.outcome.fit and b.outcome.fit) else None
    tfits = [s.outcome.fit for t in labels
             for s in [find(t, PRIMARY_OPERATOR)] if s is not None and s.outcome.fit is not None]
    t_n, t_z = maximum_pairwise_z(tfits)
    validated = (sampler_ok and primary.outcome.succeeded() and pw_n >= 2
                 and pw_z is not None and pw_z <= STABILITY_MAX_Z
                 and op_z is not None and op_z <= STABILITY_MAX_Z
                 and t_n >= 2 and t_z is not None and t_z <= STABILITY_MAX_Z)
    return ProductionSummary(chain_evidence, surfaces, sampler_ok, pw_n, pw_z, op_z, t_n, t_z, validated)


def _chain_identity_matches(campaign: "Campaign", evidence: List[ChainEvidence]) -> bool:
    """retained_chain_identity_matches (glueball_scalar_recovery_receipt.rs,
    glueball_scalar_geometry_recovery_receipt.rs:55-76)."""
    from .su3_ensemble import derive_su3_chain_seed
    expected = campaign.expected_proposals_per_chain
    if len(evidence) != campaign.chain_count:
        return False
    for k, c in enumerate(evidence):
        acc = float(c.accepts) / float(expected)
        if not (c.chain_id == k and c.derived_seed == derive_su3_chain_seed(campaign.master_seed, k)
                and c.proposals == expected and c.accepts <= c.proposals
                and MIN_ACCEPTANCE <= acc <= MAX_ACCEPTANCE and c.acceptance == acc
                and all(np.isfinite([c.plaquette, c.unitarity_residual, c.determinant_residual]))
                and 0.0 <= c.unitarity_residual <= LINK_RESIDUAL_LIMIT
                and 0.0 <= c.determinant_residual <= LINK_RESIDUAL_LIMIT):
            return False
    return True


def observed_receipt_matches(summary: ProductionSummary, campaign: "Campaign") -> bool:
    """The campaign's recorded negative receipt (glueball_scalar_production.rs:616-638,
    glueball_scalar_recovery_receipt.rs:68-91,
    glueball_scalar_geometry_recovery_receipt.rs:79-101); False for a
    campaign without one."""
    if campaign.observed_outcomes is None:
        return False
    surfaces_match = len(summary.surfaces) == len(campaign.observed_outcomes) and all(
        r.outcome.transformation == t and r.outcome.operator == o and r.outcome.fit is None
        and r.outcome.error_code == code
        for r, (t, o, code) in zip(summary.surfaces, campaign.observed_outcomes))
    return (summary.sampler_diagnostics_passed
            and (not campaign.check_chain_identity or _chain_identity_matches(campaign, summary.chain_evidence))
            and surfaces_match
            and summary.primary_window_successes == 0 and summary.primary_window_max_z is None
            and summary.operator_stability_z is None
            and summary.transformation_stability_successes == 0
            and summary.transformation_stability_max_z is None
            and not summary.scalar_pipeline_validated)


def observed_phase3f_receipt_matches(summary: ProductionSummary) -> bool:
    """glueball_scalar_production.rs:616-638."""
    return observed_receipt_matches(summary, CAMPAIGNS["phase3f"])


def observed_phase3g_receipt_matches(summary: ProductionSummary) -> bool:
    """glueball_scalar_recovery_receipt.rs:68-91."""
    return observed_receipt_matches(summary, CAMPAIGNS["phase3g"])


def observed_phase3h_receipt_matches(summary: ProductionSummary) -> bool:
    """glueball_scalar_geometry_recovery_receipt.rs:79-101."""
    return observed_receipt_matches(summary, CAMPAIGNS["phase3h"])


def run_campaign(campaign: Campaign, device: int = 0, generator_mode: str = "ordered") -> ProductionSummary:
    """One frozen campaign with its chains on the device."""
    from .ensemble import Ensemble
    from .su3_ensemble import derive_su3_chain_seed
    n = campaign.chain_count
    seeds = [derive_su3_chain_seed(campaign.master_seed, k) for k in range(n)]
    expected = campaign.expected_proposals_per_chain
    with Ensemble([list(campaign.extents)] * n, BETA, seeds, device=device) as raw:
        raw.metropolis_sweeps(PROPOSAL_ANGLE, TOTAL_SWEEPS_PER_CHAIN, generator_mode)
        prop, acc = raw.accounting()
        plaq = raw.average_plaquette()
        ures, dres = raw.max_residuals()
        evidence = []
        for k in range(n):
            if int(prop[k]) != expected or int(acc[k]) > int(prop[k]):
                raise YmError(VARIANTS["AccountingOverflow"], campaign.name)
            e = ChainEvidence(k, seeds[k], int(prop[k]), int(acc[k]), float(acc[k]) / float(prop[k]),
                              float(plaq[k]), float(ures[k]), float(dres[k]))
            if not all(np.isfinite([e.acceptance, e.plaquette, e.unitarity_residual, e.determinant_residual])):
                raise YmError(VARIANTS["NonFiniteStatistic"], campaign.name)
            if e.unitarity_residual > LINK_RESIDUAL_LIMIT or e.determinant_residual > LINK_RESIDUAL_LIMIT:
                raise YmError(VARIANTS["LinkResidualExceeded"], campaign.name)
            evidence.append(e)
        surfaces = []
        for label, kind, levels in campaign.transformations:
            if kind == "stout":
                ens = G.spatial_stout_smear(raw, G.CANONICAL_RHO, levels)
            elif kind == "block":
                ens = G.spatial_stride2_block(raw)
            else:
                ens = raw
            try:
                p, r = G.operator_samples(ens)
            finally:
                if ens is not raw:
                    ens.close()
            cp, cr = correlator_evidence(p), correlator_evidence(r)
            surfaces.append(analyze_surface(label, "plaquette-1x1", cp))
            surfaces.append(analyze_surface(label, "rectangle-2x1", cr))
    return summarize_surfaces(evidence, surfaces, campaign)


def run_production_scalar_analysis(device: int = 0, generator_mode: str = "ordered") -> ProductionSummary:
    """Phase 3F (glueball_scalar_production.rs:640-720)."""
    return run_campaign(CAMPAIGNS["phase3f"], device, generator_mode)


def run_scalar_recovery_analysis(device: int = 0, generator_mode: str = "ordered") -> ProductionSummary:
    """Phase 3G (glueball_scalar_recovery.rs:419-490): 32 fresh chains."""
    return run_campaign(CAMPAIGNS["phase3g"], device, generator_mode)


def run_scalar_geometry_recovery_analysis(device: int = 0, generator_mode: str = "ordered") -> ProductionSummary:
    """Phase 3H (glueball_scalar_geometry_recovery.rs:491-570): 6^3x10, blocked surface."""
    return run_campaign(CAMPAIGNS["phase3h"], device, generator_mode)


def run_scalar_temporal_recovery_analysis(device: int = 0, generator_mode: str = "ordered") -> ProductionSummary:
    """Phase 3I (glueball_scalar_temporal_recovery.rs:491-570): 6^3x16, 2.4e8 proposals."""
    return run_campaign(CAMPAIGNS["phase3i"], device, generator_mode)
