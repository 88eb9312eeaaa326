"""Acceptance harnesses (ymgpu.benchmarks) on synthetic chain reports, as the
reference's own tests drive them (su2_benchmark.rs:364-699,
su3_benchmark.rs tests, su3_confirmation.rs tests), plus the frozen
stream-seed goldens (su2-plaquette-baseline-v1, su3-plaquette-baseline-v1/v2).
Host code only: no GPU."""
import dataclasses

import numpy as np
import pytest

from ymgpu import benchmarks as B
from ymgpu.errors import YmError
from ymgpu.su2_ensemble import ChainReport, derive_chain_seed, diagnostics
from ymgpu.su3_ensemble import Su3ChainReport, derive_su3_chain_seed


def variant_of(fn, *args):
    with pytest.raises(YmError) as e:
        fn(*args)
    return e.value.variant


def alternating(n, lo, hi, phase=0):
    return np.array([lo if (i + phase) % 2 == 0 else hi for i in range(n)])


def drifting(n, phase):
    half = n // 2
    a = [0.601 + (0.001 if (i + phase) % 2 == 0 else -0.001) for i in range(half)]
    b = [0.603 + (0.001 if (i + phase) % 2 == 0 else -0.001) for i in range(half)]
    return np.array(a + b)


def su2_report(chain_id, meas):
    cfg = B.su2_benchmark_configs()[chain_id]
    d, _ = diagnostics(meas, B.su2.AUTOCORRELATION_MAX_LAG)
    prop = B.su2.EXPECTED_HEATBATH_UPDATES * 2
    return ChainReport(cfg, B.su2.FROZEN_CHAIN_DERIVED_SEEDS[chain_id], B.su2.EXPECTED_HEATBATH_SWEEPS,
                       B.su2.EXPECTED_OVERRELAXATION_SWEEPS, prop, B.su2.EXPECTED_HEATBATH_UPDATES,
                       B.su2.EXPECTED_HEATBATH_UPDATES / prop, np.asarray(meas), d, 0.0)


def su3_report(chain_id, meas, master=B.su3.MASTER_SEED, seeds=B.su3.FROZEN_CHAIN_DERIVED_SEEDS):
    cfg = B.su3_benchmark_configs(master, (chain_id,))[0]
    d, _ = diagnostics(meas, B.su3.AUTOCORRELATION_MAX_LAG)
    acc = B.su3.EXPECTED_PROPOSALS // 2
    return Su3ChainReport(cfg, seeds[chain_id], B.su3.EXPECTED_TOTAL_SWEEPS, B.su3.EXPECTED_PROPOSALS, acc,
                          acc / B.su3.EXPECTED_PROPOSALS, np.asarray(meas), d, 0.0, 0.0)


def test_frozen_stream_seeds_match_the_reference_goldens(golden):
    v2 = golden["su2-plaquette-baseline-v1.json"]
    for cid, seed in zip(B.su2.CHAIN_IDS, B.su2.FROZEN_CHAIN_DERIVED_SEEDS):
        assert derive_chain_seed(B.su2.MASTER_SEED, cid) == seed
    for cid, seed in zip(B.su3.CHAIN_IDS, B.su3.FROZEN_CHAIN_DERIVED_SEEDS):
        assert derive_su3_chain_seed(B.su3.MASTER_SEED, cid) == seed
    for cid, seed in zip(B.su3.CONFIRMATION_CHAIN_IDS, B.su3.CONFIRMATION_DERIVED_SEEDS):
        assert derive_su3_chain_seed(B.su3.CONFIRMATION_MASTER_SEED, cid) == seed
    two = [v for v in v2["vectors"] if v["id"] == "two-independent-chain-comparison"][0]
    assert int(two["master_seed"], 16) == B.su2.MASTER_SEED
    assert two["measurements_per_chain"] == B.su2.MEASUREMENTS
    assert two["thermalization_sweeps"] == B.su2.THERMALIZATION_SWEEPS
    env = [v for v in v2["vectors"] if v["id"] == "published-source-envelope"][0]["expected_interval"]
    assert env == [B.su2.SOURCE_ENVELOPE_MIN, B.su2.SOURCE_ENVELOPE_MAX]
    assert B.su2.EXPECTED_HEATBATH_UPDATES == 3_520_000
    assert B.su2.MAX_EXPECTED_HEATBATH_PROPOSALS == 35_200_000_000


def test_su2_summary_gates():
    n = B.su2.MEASUREMENTS
    ok = B.su2_summarize_two_chains(su2_report(0, alternating(n, 0.601, 0.603)),
                                    su2_report(1, alternating(n, 0.601, 0.603, 1)))
    assert ok.source_envelope_reproduced and ok.diagnostics_trustworthy
    assert ok.phase2_graduation_gate_satisfied
    drift = B.su2_summarize_two_chains(su2_report(0, drifting(n, 0)), su2_report(1, drifting(n, 1)))
    assert drift.source_envelope_reproduced and drift.chain_consistency_z == 0.0
    assert drift.min_effective_sample_size >= B.su2.MIN_CHAIN_ESS
    assert B.su2.MAX_STATIONARITY_Z < drift.max_stationarity_z < 50.0
    assert not drift.diagnostics_trustworthy and not drift.phase2_graduation_gate_satisfied
    # statistics are recomputed from the retained series, not the cached diagnostics
    a = su2_report(0, alternating(n, 0.899, 0.901))
    b = su2_report(1, alternating(n, 0.8985, 0.9015))
    cached, _ = diagnostics(alternating(n, 0.601, 0.603), B.su2.AUTOCORRELATION_MAX_LAG)
    s = B.su2_summarize_two_chains(dataclasses.replace(a, diagnostics=cached),
                                   dataclasses.replace(b, diagnostics=cached))
    assert s.chain_means[0] > 0.89 and not s.source_envelope_reproduced


def test_su2_summary_fails_closed():
    n = B.su2.MEASUREMENTS
    a, b = su2_report(0, alternating(n, 0.601, 0.603)), su2_report(1, alternating(n, 0.601, 0.603, 1))
    S = B.su2_summarize_two_chains
    assert variant_of(S, b, a) == "WrongBenchmarkConfiguration"
    assert variant_of(S, dataclasses.replace(a, sampler_id="X"), b) == "WrongBenchmarkConfiguration"
    assert variant_of(S, a, dataclasses.replace(b, measurements=a.measurements)) == \
        "DuplicateMeasurementSeries"
    bad = a.measurements.copy()
    bad[3] = 1.5
    assert variant_of(S, dataclasses.replace(a, measurements=bad), b) == "InvalidPlaquetteSample"
    assert variant_of(S, dataclasses.replace(a, heatbath_proposals=0, heatbath_updates=0,
                                             mean_heatbath_acceptance=0.0), b) == "InvalidHeatbathAccounting"
    assert variant_of(S, dataclasses.replace(a, mean_heatbath_acceptance=0.4), b) == "InvalidAcceptanceEvidence"
    assert variant_of(S, a, dataclasses.replace(b, final_link_unit_residual=-1.0)) == "InvalidLinkUnitResidual"
    flat = su2_report(0, np.full(n, 0.602)), su2_report(1, np.full(n, 0.603))
    assert variant_of(S, *flat) == "StationarityDiagnosticFailed"
    assert variant_of(B.su2_stationarity_diagnostic, np.full(n, 0.602)) == "StationarityDiagnosticFailed"
    assert variant_of(B.su2_stationarity_diagnostic, np.full(n - 1, 0.602)) == "WrongBenchmarkConfiguration"


def test_su3_two_chain_and_confirmation_gates():
    n = B.su3.MEASUREMENTS
    a, b = su3_report(0, alternating(n, 0.59, 0.594)), su3_report(1, alternating(n, 0.59, 0.594, 1))
    s = B.su3_summarize_two_chains(a, b)
    assert s.published_su3_baseline_reproduced and s.chain_acceptances == (0.5, 0.5)
    S = B.su3_summarize_two_chains
    assert variant_of(S, a, dataclasses.replace(b, derived_seed=a.derived_seed)) == "DuplicateChainIdentity"
    assert variant_of(S, dataclasses.replace(a, metropolis_proposals=1), b) == "InvalidMetropolisAccounting"
    low = dataclasses.replace(a, metropolis_accepts=1, mean_metropolis_acceptance=1 / B.su3.EXPECTED_PROPOSALS)
    assert variant_of(S, low, b) == "InvalidAcceptanceEvidence"
    assert variant_of(S, a, dataclasses.replace(b, final_link_determinant_residual=np.nan)) == \
        "InvalidLinkResidual"
    assert variant_of(S, dataclasses.replace(a, total_sweeps=1), b) == "WrongBenchmarkConfiguration"
    seeds = B.su3.CONFIRMATION_DERIVED_SEEDS
    four = [su3_report(k, alternating(n, 0.585 + 0.001 * k, 0.595 + 0.001 * k, k % 2),
                       B.su3.CONFIRMATION_MASTER_SEED, seeds) for k in range(4)]
    c = B.summarize_four_chains(four)
    assert c.aggregate_effective_sample_size >= B.su3.MIN_AGGREGATE_ESS
    assert c.source_envelope_reproduced
    assert abs(c.pooled_mean - np.mean([f.measurements.mean() for f in four])) < 1e-12
    assert variant_of(B.summarize_four_chains, four[:3] + [four[0]]) == "DuplicateChainIdentity"
    assert variant_of(B.summarize_four_chains, [four[1], four[0]] + four[2:]) == "WrongBenchmarkConfiguration"
