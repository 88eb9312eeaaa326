"""Published-baseline acceptance harnesses -- mirror of the reference modules
``su2_benchmark`` (phase 2B, two SU(2) 10^4 chains at beta 2.3),
``su3_benchmark`` (phase 2C2, two SU(3) 4^4 chains at beta 6.0) and
``su3_confirmation`` (four SU(3) chains, a second master seed).

The summaries recompute every statistic from the retained measurement
series with the reference's chain diagnostics (libymgpu host FP64), apply
the reference's frozen gates in the reference's order, and report whether
the published plaquette envelope is reproduced.  ``run_*`` build the frozen
chain configurations, run them on the device through ``run_chains`` and
summarise them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Sequence

from .errors import VARIANTS, YmError
from .su2_ensemble import diagnostics


def _fail(name: str, where: str) -> YmError:
    return YmError(VARIANTS[name], where)


def _finite(*xs) -> bool:
    return all(math.isfinite(x) for x in xs)


@dataclass(frozen=True)
class StationarityDiagnostic:
    first_half_mean: float
    second_half_mean: float
    first_half_standard_error: float
    second_half_standard_error: float
    drift_z: float


def _is_constant(values) -> bool:
    return len(values) > 0 and all(v == values[0] for v in values[1:])


def _stationarity(values, measurements: int, max_lag: int) -> StationarityDiagnostic:
    """stationarity_diagnostic (su2_benchmark.rs:192-237, su3_benchmark.rs:192-237):
    drift z of the two halves' means with autocorrelation-aware errors."""
    half = measurements // 2
    if len(values) != measurements or half * 2 != measurements or max_lag >= half:
        raise _fail("WrongBenchmarkConfiguration", "stationarity_diagnostic")
    a, b = [float(v) for v in values[:half]], [float(v) for v in values[half:]]
    if _is_constant(a) or _is_constant(b):
        raise _fail("StationarityDiagnosticFailed", "stationarity_diagnostic")
    try:
        first, _ = diagnostics(a, max_lag)
        second, _ = diagnostics(b, max_lag)
    except YmError:
        raise _fail("StationarityDiagnosticFailed", "stationarity_diagnostic") from None
    if first.variance == 0.0 or second.variance == 0.0:
        raise _fail("StationarityDiagnosticFailed", "stationarity_diagnostic")
    diff = abs(first.mean - second.mean)
    scale = math.sqrt(first.standard_error * first.standard_error +
                      second.standard_error * second.standard_error)
    if scale == 0.0:
        raise _fail("StationarityDiagnosticFailed", "stationarity_diagnostic")
    z = diff / scale
    if not _finite(first.mean, second.mean, first.standard_error, second.standard_error, z):
        raise _fail("NonFiniteStatistic", "stationarity_diagnostic")
    return StationarityDiagnostic(first.mean, second.mean, first.standard_error,
                                  second.standard_error, z)


def _physical(values, lower: float, upper: float) -> bool:
    return all(math.isfinite(v) and lower <= v <= upper for v in values)


def _same_series(a, b) -> bool:
    return len(a) == len(b) and all(x == y for x, y in zip(a, b))


def _pair_z(m0, m1, s0, s1) -> float:
    diff = abs(m0 - m1)
    scale = math.sqrt(s0 * s0 + s1 * s1)
    if scale == 0.0:
        return 0.0 if diff == 0.0 else math.inf
    return diff / scale


# ============================================================ SU(2), phase 2B
class su2:
    """su2_benchmark.rs:19-52."""
    BENCHMARK_ID = "YM-SU2-PLAQUETTE-BASELINE-V1"
    PRIMARY_DOI = "10.1103/PhysRevLett.109.111601"
    BETA = 2.3
    EXTENTS = (10, 10, 10, 10)
    SOURCE_ENVELOPE_MIN = 0.59
    SOURCE_ENVELOPE_MAX = 0.62
    MASTER_SEED = 0x2B00_2012_1116_0101
    CHAIN_IDS = (0, 1)
    FROZEN_PHASE2A_SAMPLER_ID = "YM-SU2-ENSEMBLE-V1"
    FROZEN_PHASE2A_RNG_ID = "SPLITMIX64-V1"
    FROZEN_CHAIN_DERIVED_SEEDS = (0x044D_F781_F86A_2ADE, 0x4EBD_9478_3D50_8D2E)
    THERMALIZATION_SWEEPS = 40
    MEASUREMENTS = 48
    SWEEPS_BETWEEN_MEASUREMENTS = 1
    OVERRELAXATION_SWEEPS_PER_HEATBATH = 1
    MAX_HEATBATH_ATTEMPTS_PER_LINK = 10_000
    AUTOCORRELATION_MAX_LAG = 12
    MIN_CHAIN_ESS = 6.0
    MAX_CHAIN_CONSISTENCY_Z = 5.0
    STATIONARITY_AUTOCORRELATION_MAX_LAG = 6
    MAX_STATIONARITY_Z = 5.0
    MAX_LINK_UNIT_RESIDUAL = 1.0e-12
    PLAQUETTE_SAMPLE_TOLERANCE = 1.0e-12
    LINKS_PER_HEATBATH_SWEEP = 10 ** 4 * 4
    EXPECTED_HEATBATH_SWEEPS = THERMALIZATION_SWEEPS + MEASUREMENTS * SWEEPS_BETWEEN_MEASUREMENTS
    EXPECTED_OVERRELAXATION_SWEEPS = EXPECTED_HEATBATH_SWEEPS * OVERRELAXATION_SWEEPS_PER_HEATBATH
    EXPECTED_HEATBATH_UPDATES = LINKS_PER_HEATBATH_SWEEP * EXPECTED_HEATBATH_SWEEPS
    MAX_EXPECTED_HEATBATH_PROPOSALS = EXPECTED_HEATBATH_UPDATES * MAX_HEATBATH_ATTEMPTS_PER_LINK


@dataclass(frozen=True)
class Su2BenchmarkSummary:
    chain_means: tuple
    chain_standard_errors: tuple
    chain_effective_sample_sizes: tuple
    stationarity: tuple
    max_stationarity_z: float
    pooled_mean: float
    pooled_standard_error: float
    chain_consistency_z: float
    min_effective_sample_size: float
    max_link_unit_residual: float
    source_envelope_reproduced: bool
    diagnostics_trustworthy: bool
    phase2_graduation_gate_satisfied: bool


def su2_stationarity_diagnostic(values) -> StationarityDiagnostic:
    return _stationarity(values, su2.MEASUREMENTS, su2.STATIONARITY_AUTOCORRELATION_MAX_LAG)


def _su2_matches(report, chain_id: int) -> bool:   # su2_benchmark.rs:137-158
    if chain_id not in su2.CHAIN_IDS:
        return False
    c = report.config
    return (report.sampler_id == su2.FROZEN_PHASE2A_SAMPLER_ID
            and report.rng_id == su2.FROZEN_PHASE2A_RNG_ID
            and report.derived_seed == su2.FROZEN_CHAIN_DERIVED_SEEDS[su2.CHAIN_IDS.index(chain_id)]
            and tuple(c.extents) == su2.EXTENTS and c.beta == su2.BETA
            and c.master_seed == su2.MASTER_SEED and c.chain_id == chain_id
            and c.thermalization_sweeps == su2.THERMALIZATION_SWEEPS
            and c.measurements == su2.MEASUREMENTS
            and len(report.measurements) == su2.MEASUREMENTS
            and c.sweeps_between_measurements == su2.SWEEPS_BETWEEN_MEASUREMENTS
            and c.overrelaxation_sweeps_per_heatbath == su2.OVERRELAXATION_SWEEPS_PER_HEATBATH
            and c.max_heatbath_attempts_per_link == su2.MAX_HEATBATH_ATTEMPTS_PER_LINK
            and c.autocorrelation_max_lag == su2.AUTOCORRELATION_MAX_LAG)


def _su2_acceptance(report) -> float:   # su2_benchmark.rs:169-185
    if (report.total_heatbath_sweeps != su2.EXPECTED_HEATBATH_SWEEPS
            or report.total_overrelaxation_sweeps != su2.EXPECTED_OVERRELAXATION_SWEEPS
            or report.heatbath_updates != su2.EXPECTED_HEATBATH_UPDATES
            or report.heatbath_proposals < su2.EXPECTED_HEATBATH_UPDATES
            or report.heatbath_proposals > su2.MAX_EXPECTED_HEATBATH_PROPOSALS):
        raise _fail("InvalidHeatbathAccounting", "summarize_two_chains")
    acc = float(report.heatbath_updates) / float(report.heatbath_proposals)
    if not math.isfinite(acc) or acc <= 0.0 or acc > 1.0 or report.mean_heatbath_acceptance != acc:
        raise _fail("InvalidAcceptanceEvidence", "summarize_two_chains")
    return acc


def su2_summarize_two_chains(first, second) -> Su2BenchmarkSummary:
    """summarize_two_chains (su2_benchmark.rs:239-362)."""
    where = "su2_summarize_two_chains"
    if not _su2_matches(first, su2.CHAIN_IDS[0]) or not _su2_matches(second, su2.CHAIN_IDS[1]):
        raise _fail("WrongBenchmarkConfiguration", where)
    if first.derived_seed == second.derived_seed:
        raise _fail("DuplicateChainIdentity", where)
    if _same_series(first.measurements, second.measurements):
        raise _fail("DuplicateMeasurementSeries", where)
    lo, hi = -1.0 - su2.PLAQUETTE_SAMPLE_TOLERANCE, 1.0 + su2.PLAQUETTE_SAMPLE_TOLERANCE
    if not _physical(first.measurements, lo, hi) or not _physical(second.measurements, lo, hi):
        raise _fail("InvalidPlaquetteSample", where)
    _su2_acceptance(first)
    _su2_acceptance(second)
    for r in (first, second):
        if not math.isfinite(r.final_link_unit_residual) or r.final_link_unit_residual < 0.0:
            raise _fail("InvalidLinkUnitResidual", where)
    try:
        d = [diagnostics(r.measurements, su2.AUTOCORRELATION_MAX_LAG)[0] for r in (first, second)]
    except YmError:
        raise _fail("NonFiniteStatistic", where) from None
    means = (d[0].mean, d[1].mean)
    ses = (d[0].standard_error, d[1].standard_error)
    ess = (d[0].effective_sample_size, d[1].effective_sample_size)
    st = (su2_stationarity_diagnostic(first.measurements), su2_stationarity_diagnostic(second.measurements))
    max_z = max(st[0].drift_z, st[1].drift_z)
    if not _finite(*means, *ses, *ess, max_z):
        raise _fail("NonFiniteStatistic", where)
    pooled = 0.5 * (means[0] + means[1])
    pooled_se = 0.5 * math.sqrt(ses[0] * ses[0] + ses[1] * ses[1])
    cz = _pair_z(means[0], means[1], ses[0], ses[1])
    min_ess = min(ess)
    max_res = max(first.final_link_unit_residual, second.final_link_unit_residual)
    if not _finite(pooled, pooled_se, cz, min_ess, max_res):
        raise _fail("NonFiniteStatistic", where)
    env = su2.SOURCE_ENVELOPE_MIN <= pooled <= su2.SOURCE_ENVELOPE_MAX
    trust = (min_ess >= su2.MIN_CHAIN_ESS and cz <= su2.MAX_CHAIN_CONSISTENCY_Z
             and max_z <= su2.MAX_STATIONARITY_Z and max_res <= su2.MAX_LINK_UNIT_RESIDUAL)
    return Su2BenchmarkSummary(means, ses, ess, st, max_z, pooled, pooled_se, cz, min_ess, max_res,
                               env, trust, env and trust)


def su2_benchmark_configs():
    from .su2_ensemble import EnsembleConfig
    return [EnsembleConfig(su2.EXTENTS, su2.BETA, su2.MASTER_SEED, cid, su2.THERMALIZATION_SWEEPS,
                           su2.MEASUREMENTS, su2.SWEEPS_BETWEEN_MEASUREMENTS,
                           su2.OVERRELAXATION_SWEEPS_PER_HEATBATH, su2.MAX_HEATBATH_ATTEMPTS_PER_LINK,
                           su2.AUTOCORRELATION_MAX_LAG) for cid in su2.CHAIN_IDS]


def run_su2_benchmark(device: int = 0) -> Su2BenchmarkSummary:
    """Both frozen phase-2B chains on the device, summarised."""
    from .su2_ensemble import run_chains
    a, b = run_chains(su2_benchmark_configs(), device=device)
    return su2_summarize_two_chains(a, b)


# ============================================================ SU(3), phase 2C2
class su3:
    """su3_benchmark.rs:23-53 (and su3_confirmation.rs:29-39)."""
    BENCHMARK_ID = "YM-SU3-PLAQUETTE-BASELINE-V1"
    PRIMARY_DOI = "10.1088/0305-4616/7/5/001"
    BETA = 6.0
    EXTENTS = (4, 4, 4, 4)
    SOURCE_ENVELOPE_MIN = 0.56
    SOURCE_ENVELOPE_MAX = 0.63
    MASTER_SEED = 0x2C02_1981_0501_0001
    CHAIN_IDS = (0, 1)
    FROZEN_CHAIN_DERIVED_SEEDS = (0x2FF3_BF48_550D_1457, 0xEF76_36A5_6E8E_A29A)
    PROPOSAL_ANGLE = 0.35
    THERMALIZATION_SWEEPS = 192
    MEASUREMENTS = 128
    SWEEPS_BETWEEN_MEASUREMENTS = 2
    AUTOCORRELATION_MAX_LAG = 24
    MIN_CHAIN_ESS = 8.0
    MAX_CHAIN_CONSISTENCY_Z = 5.0
    STATIONARITY_AUTOCORRELATION_MAX_LAG = 12
    MAX_STATIONARITY_Z = 5.0
    MIN_METROPOLIS_ACCEPTANCE = 0.10
    MAX_METROPOLIS_ACCEPTANCE = 0.95
    MAX_LINK_UNITARITY_RESIDUAL = 5.0e-12
    MAX_LINK_DETERMINANT_RESIDUAL = 5.0e-12
    PLAQUETTE_SAMPLE_TOLERANCE = 1.0e-12
    ACCEPTANCE_EVIDENCE_TOLERANCE = 1.0e-12
    LINKS_PER_SWEEP = 4 ** 4 * 4
    PROPOSALS_PER_LINK_PER_SWEEP = 8
    EXPECTED_TOTAL_SWEEPS = THERMALIZATION_SWEEPS + MEASUREMENTS * SWEEPS_BETWEEN_MEASUREMENTS
    EXPECTED_PROPOSALS = LINKS_PER_SWEEP * PROPOSALS_PER_LINK_PER_SWEEP * EXPECTED_TOTAL_SWEEPS
    CONFIRMATION_ID = "YM-SU3-PLAQUETTE-BASELINE-V2"
    CONFIRMATION_MASTER_SEED = 0x2C02_1981_0501_0002
    CONFIRMATION_CHAIN_IDS = (0, 1, 2, 3)
    CONFIRMATION_DERIVED_SEEDS = (0xDFCD_AB17_9476_617A, 0x151D_D841_CCEF_81C6,
                                  0x9C28_EDED_CA3D_1AE2, 0x17DB_BF4A_0021_4611)
    MIN_AGGREGATE_ESS = 16.0
    MAX_PAIRWISE_CHAIN_CONSISTENCY_Z = 5.0


@dataclass(frozen=True)
class Su3BenchmarkSummary:
    chain_means: tuple
    chain_standard_errors: tuple
    chain_effective_sample_sizes: tuple
    chain_acceptances: tuple
    stationarity: tuple
    max_stationarity_z: float
    pooled_mean: float
    pooled_standard_error: float
    chain_consistency_z: float
    min_effective_sample_size: float
    max_link_unitarity_residual: float
    max_link_determinant_residual: float
    source_envelope_reproduced: bool
    diagnostics_trustworthy: bool
    published_su3_baseline_reproduced: bool


@dataclass(frozen=True)
class ConfirmationSummary:
    chain_means: tuple
    chain_standard_errors: tuple
    chain_effective_sample_sizes: tuple
    chain_acceptances: tuple
    stationarity: tuple
    max_stationarity_z: float
    pooled_mean: float
    pooled_standard_error: float
    aggregate_effective_sample_size: float
    max_pairwise_chain_consistency_z: float
    max_link_unitarity_residual: float
    max_link_determinant_residual: float
    source_envelope_reproduced: bool
    diagnostics_trustworthy: bool
    published_su3_baseline_reproduced: bool


def su3_stationarity_diagnostic(values) -> StationarityDiagnostic:
    return _stationarity(values, su3.MEASUREMENTS, su3.STATIONARITY_AUTOCORRELATION_MAX_LAG)


def _su3_matches(report, chain_id: int, master_seed: int, ids, seeds) -> bool:
    from .su3_ensemble import PROPOSAL_ID, RNG_ID, SAMPLER_ID, STREAM_ID
    if chain_id not in ids:
        return False
    c = report.config
    return (report.sampler_id == SAMPLER_ID and report.proposal_id == PROPOSAL_ID
            and report.rng_id == RNG_ID and report.stream_id == STREAM_ID
            and report.derived_seed == seeds[ids.index(chain_id)]
            and tuple(c.extents) == su3.EXTENTS and c.beta == su3.BETA
            and c.master_seed == master_seed and c.chain_id == chain_id
            and c.thermalization_sweeps == su3.THERMALIZATION_SWEEPS
            and c.measurements == su3.MEASUREMENTS
            and len(report.measurements) == su3.MEASUREMENTS
            and c.sweeps_between_measurements == su3.SWEEPS_BETWEEN_MEASUREMENTS
            and c.proposal_angle == su3.PROPOSAL_ANGLE
            and c.autocorrelation_max_lag == su3.AUTOCORRELATION_MAX_LAG
            and report.total_sweeps == su3.EXPECTED_TOTAL_SWEEPS)


def _su3_acceptance(report, where: str) -> float:   # su3_benchmark.rs:168-184
    if (report.metropolis_proposals != su3.EXPECTED_PROPOSALS or report.metropolis_accepts == 0
            or report.metropolis_accepts > report.metropolis_proposals):
        raise _fail("InvalidMetropolisAccounting", where)
    acc = float(report.metropolis_accepts) / float(report.metropolis_proposals)
    if (not math.isfinite(acc) or not math.isfinite(report.mean_metropolis_acceptance)
            or abs(report.mean_metropolis_acceptance - acc) > su3.ACCEPTANCE_EVIDENCE_TOLERANCE
            or not su3.MIN_METROPOLIS_ACCEPTANCE <= acc <= su3.MAX_METROPOLIS_ACCEPTANCE):
        raise _fail("InvalidAcceptanceEvidence", where)
    return acc


def _su3_residuals_ok(r) -> bool:
    return (math.isfinite(r.final_link_unitarity_residual)
            and math.isfinite(r.final_link_determinant_residual)
            and r.final_link_unitarity_residual >= 0.0 and r.final_link_determinant_residual >= 0.0)


def su3_summarize_two_chains(first, second) -> Su3BenchmarkSummary:
    """summarize_two_chains (su3_benchmark.rs:239-360)."""
    where = "su3_summarize_two_chains"
    if first.derived_seed == second.derived_seed:
        raise _fail("DuplicateChainIdentity", where)
    m = lambda r, cid: _su3_matches(r, cid, su3.MASTER_SEED, su3.CHAIN_IDS, su3.FROZEN_CHAIN_DERIVED_SEEDS)
    if not m(first, 0) or not m(second, 1):
        raise _fail("WrongBenchmarkConfiguration", where)
    if _same_series(first.measurements, second.measurements):
        raise _fail("DuplicateMeasurementSeries", where)
    lo, hi = -0.5 - su3.PLAQUETTE_SAMPLE_TOLERANCE, 1.0 + su3.PLAQUETTE_SAMPLE_TOLERANCE
    if not _physical(first.measurements, lo, hi) or not _physical(second.measurements, lo, hi):
        raise _fail("InvalidPlaquetteSample", where)
    accs = (_su3_acceptance(first, where), _su3_acceptance(second, where))
    if not _su3_residuals_ok(first) or not _su3_residuals_ok(second):
        raise _fail("InvalidLinkResidual", where)
    try:
        d = [diagnostics(r.measurements, su3.AUTOCORRELATION_MAX_LAG)[0] for r in (first, second)]
    except YmError:
        raise _fail("NonFiniteStatistic", where) from None
    means = (d[0].mean, d[1].mean)
    ses = (d[0].standard_error, d[1].standard_error)
    ess = (d[0].effective_sample_size, d[1].effective_sample_size)
    st = (su3_stationarity_diagnostic(first.measurements), su3_stationarity_diagnostic(second.measurements))
    max_z = max(st[0].drift_z, st[1].drift_z)
    pooled = 0.5 * (means[0] + means[1])
    pooled_se = 0.5 * math.sqrt(ses[0] * ses[0] + ses[1] * ses[1])
    cz = _pair_z(means[0], means[1], ses[0], ses[1])
    min_ess = min(ess)
    max_u = max(first.final_link_unitarity_residual, second.final_link_unitarity_residual)
    max_d = max(first.final_link_determinant_residual, second.final_link_determinant_residual)
    if not _finite(*means, *ses, *ess, *accs, max_z, pooled, pooled_se, cz, min_ess, max_u, max_d):
        raise _fail("NonFiniteStatistic", where)
    env = su3.SOURCE_ENVELOPE_MIN <= pooled <= su3.SOURCE_ENVELOPE_MAX
    trust = (min_ess >= su3.MIN_CHAIN_ESS and cz <= su3.MAX_CHAIN_CONSISTENCY_Z
             and max_z <= su3.MAX_STATIONARITY_Z and max_u <= su3.MAX_LINK_UNITARITY_RESIDUAL
             and max_d <= su3.MAX_LINK_DETERMINANT_RESIDUAL)
    return Su3BenchmarkSummary(means, ses, ess, accs, st, max_z, pooled, pooled_se, cz, min_ess,
                               max_u, max_d, env, trust, env and trust)


def summarize_four_chains(reports: Sequence) -> ConfirmationSummary:
    """summarize_four_chains (su3_confirmation.rs:127-260)."""
    where = "summarize_four_chains"
    if len(reports) != 4:
        raise _fail("WrongBenchmarkConfiguration", where)
    for i in range(4):
        for j in range(i + 1, 4):
            if reports[i].derived_seed == reports[j].derived_seed:
                raise _fail("DuplicateChainIdentity", where)
            if _same_series(reports[i].measurements, reports[j].measurements):
                raise _fail("DuplicateMeasurementSeries", where)
    lo, hi = -0.5 - su3.PLAQUETTE_SAMPLE_TOLERANCE, 1.0 + su3.PLAQUETTE_SAMPLE_TOLERANCE
    for i, r in enumerate(reports):
        if not _su3_matches(r, su3.CONFIRMATION_CHAIN_IDS[i], su3.CONFIRMATION_MASTER_SEED,
                            su3.CONFIRMATION_CHAIN_IDS, su3.CONFIRMATION_DERIVED_SEEDS):
            raise _fail("WrongBenchmarkConfiguration", where)
        if not _physical(r.measurements, lo, hi):
            raise _fail("InvalidPlaquetteSample", where)
        if not _su3_residuals_ok(r):
            raise _fail("InvalidLinkResidual", where)
    accs = tuple(_su3_acceptance(r, where) for r in reports)
    try:
        d = [diagnostics(r.measurements, su3.AUTOCORRELATION_MAX_LAG)[0] for r in reports]
    except YmError:
        raise _fail("NonFiniteStatistic", where) from None
    means = tuple(x.mean for x in d)
    ses = tuple(x.standard_error for x in d)
    ess = tuple(x.effective_sample_size for x in d)
    if (not _finite(*means) or not all(math.isfinite(s) and s > 0.0 for s in ses)
            or not all(math.isfinite(e) and e > 0.0 for e in ess) or not _finite(*accs)):
        raise _fail("NonFiniteStatistic", where)
    st = tuple(su3_stationarity_diagnostic(r.measurements) for r in reports)
    max_z = 0.0
    for s in st:
        max_z = max(max_z, s.drift_z)
    total = 0.0
    for x in means:
        total += x
    pooled = total / 4.0
    sq = 0.0
    for s in ses:
        sq += s * s
    pooled_se = math.sqrt(sq) / 4.0
    agg = 0.0
    for e in ess:
        agg += e
    max_pair = 0.0
    for i in range(4):
        for j in range(i + 1, 4):
            diff = abs(means[i] - means[j])
            scale = math.sqrt(ses[i] * ses[i] + ses[j] * ses[j])
            if not math.isfinite(diff) or not math.isfinite(scale) or scale <= 0.0:
                raise _fail("NonFiniteStatistic", where)
            max_pair = max(max_pair, diff / scale)
    max_u = max([0.0] + [r.final_link_unitarity_residual for r in reports])
    max_d = max([0.0] + [r.final_link_determinant_residual for r in reports])
    if not _finite(max_z, pooled, pooled_se, agg, max_pair, max_u, max_d):
        raise _fail("NonFiniteStatistic", where)
    env = su3.SOURCE_ENVELOPE_MIN <= pooled <= su3.SOURCE_ENVELOPE_MAX
    trust = (agg >= su3.MIN_AGGREGATE_ESS and max_pair <= su3.MAX_PAIRWISE_CHAIN_CONSISTENCY_Z
             and max_z <= su3.MAX_STATIONARITY_Z and max_u <= su3.MAX_LINK_UNITARITY_RESIDUAL
             and max_d <= su3.MAX_LINK_DETERMINANT_RESIDUAL)
    return ConfirmationSummary(means, ses, ess, accs, st, max_z, pooled, pooled_se, agg, max_pair,
                               max_u, max_d, env, trust, env and trust)


def su3_benchmark_configs(master_seed: int = su3.MASTER_SEED, chain_ids=su3.CHAIN_IDS):
    from .su3_ensemble import Su3EnsembleConfig
    return [Su3EnsembleConfig(su3.EXTENTS, su3.BETA, master_seed, cid, su3.THERMALIZATION_SWEEPS,
                              su3.MEASUREMENTS, su3.SWEEPS_BETWEEN_MEASUREMENTS, su3.PROPOSAL_ANGLE,
                              su3.AUTOCORRELATION_MAX_LAG) for cid in chain_ids]


def run_su3_benchmark(device: int = 0) -> Su3BenchmarkSummary:
    """Both frozen phase-2C2 chains on the device, summarised."""
    from .su3_ensemble import run_chains
    a, b = run_chains(su3_benchmark_configs(), device=device)
    return su3_summarize_two_chains(a, b)


def run_su3_confirmation(device: int = 0) -> ConfirmationSummary:
    """The four frozen confirmation chains on the device, summarised."""
    from .su3_ensemble import run_chains
    reports = run_chains(su3_benchmark_configs(su3.CONFIRMATION_MASTER_SEED,
                                               su3.CONFIRMATION_CHAIN_IDS), device=device)
    return summarize_four_chains(reports)
