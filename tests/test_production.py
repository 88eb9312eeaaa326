"""Phase-3F production-campaign logic (ymgpu.production) on host inputs:
frozen schedule against glueball-scalar-production-phase3f-v1, the
scientific error codes, surface analysis, stability gates and the observed
receipt rule (glueball_scalar_production.rs:474-638).  No GPU."""
import dataclasses
import math

import numpy as np
import pytest

from ymgpu import analysis as A
from ymgpu import production as P


def test_frozen_schedule_matches_the_vector(golden):
    vs = {v["id"]: v for v in golden["glueball-scalar-production-phase3f-v1.json"]["vectors"]}
    s = vs["predeclared-independent-chain-production-schedule"]
    assert tuple(s["extents"]) == P.EXTENTS and s["beta"] == P.BETA
    assert int(s["master_seed_hex"], 16) == P.MASTER_SEED and s["chain_count"] == P.CHAIN_COUNT
    assert s["thermalization_sweeps"] == P.THERMALIZATION_SWEEPS
    assert s["post_thermalization_sweeps"] == P.POST_THERMALIZATION_SWEEPS
    assert s["proposal_angle"] == P.PROPOSAL_ANGLE
    assert s["expected_proposals_per_chain"] == P.EXPECTED_PROPOSALS_PER_CHAIN
    w = vs["predeclared-fit-windows"]
    assert [[x.start, x.end] for x in P.CANDIDATE_WINDOWS] == w["candidate_windows"]
    assert w["primary_surface"] == f"{P.PRIMARY_TRANSFORMATION}/{P.PRIMARY_OPERATOR}"
    scan = vs["predeclared-operator-transformation-scan"]
    assert tuple(scan["operators"]) == P.OPERATORS and tuple(scan["transformations"]) == P.TRANSFORMATION_LABELS
    rec = vs["observed-negative-production-receipt"]
    assert [(o["transformation"], o["operator"], o["reason"]) for o in rec["surface_outcomes"]] == \
        list(P.OBSERVED_SURFACE_OUTCOMES)


def test_scientific_codes_and_surface_analysis():
    assert P.scientific_fit_error_code("AcoshDomainViolation") == P.OBSERVED_REJECTION_CODE
    assert P.scientific_fit_error_code("NoAcceptedPlateauWindow") == "no-accepted-plateau-window"
    assert P.scientific_fit_error_code("TooFewJackknifeReplicates") is None
    # a clean single-state correlator (16 replicas) is fitted
    rng = np.random.default_rng(7)
    full = A.analytic_periodic_single_state(10, 0.8, 1.0)
    jk = [full * (1.0 + 0.01 * rng.standard_normal(10)) for _ in range(16)]
    rec = P.analyze_surface("stout-2", "plaquette-1x1", P.CorrelatorEvidence(full, jk))
    assert rec.outcome.succeeded() and abs(rec.outcome.fit.fitted_mass - 0.8) < 0.05
    # noise-dominated: the effective mass is rejected, recorded as an outcome
    noisy = P.CorrelatorEvidence(np.array([1.0, 0.1, -0.05, 0.02, 0.01, 0.0, 0.01, 0.02, -0.05, 0.1]),
                                 [np.array([1.0, 0.1, -0.05, 0.02, 0.01, 0.0, 0.01, 0.02, -0.05, 0.1]) +
                                  0.001 * k for k in range(16)])
    rec = P.analyze_surface("raw", "plaquette-1x1", noisy)
    assert not rec.outcome.succeeded() and rec.outcome.error_code == P.OBSERVED_REJECTION_CODE


def _fit(mass, se):
    return A.ScalarFitResult(10, 16, A.FitWindow(1, 3), mass, 1.0, mass, 1.0, 1.0, 1, 1.0, mass, se, 1.0,
                             0.1, 0.2)


def test_stability_gates_and_receipt():
    z = P.stable_z(_fit(0.8, 0.03), _fit(0.7, 0.04))
    assert abs(z - 0.1 / 0.05) < 1e-12
    assert P.stable_z(_fit(0.8, 0.0), _fit(0.7, 0.0)) is None
    assert P.maximum_pairwise_z([_fit(0.8, 0.03)]) == (1, None)
    n, mz = P.maximum_pairwise_z([_fit(0.8, 0.03), _fit(0.7, 0.04), _fit(0.75, 0.04)])
    assert n == 3 and abs(mz - 2.0) < 1e-12
    ev = [P.ChainEvidence(k, k, P.EXPECTED_PROPOSALS_PER_CHAIN, 1, 0.5, 0.5, 0.0, 0.0) for k in range(16)]
    base = np.array([1.0, 0.1, -0.05, 0.02, 0.01, 0.0, 0.01, 0.02, -0.05, 0.1])
    dummy = P.CorrelatorEvidence(base, [base + 0.001 * k for k in range(16)])   # rejected in every window
    rejected = [P.SurfaceRecord(P.SurfaceOutcome(t, o, None, c), dummy) for t, o, c in P.OBSERVED_SURFACE_OUTCOMES]
    s = P.summarize_surfaces(ev, rejected)
    assert P.observed_phase3f_receipt_matches(s) and not s.scalar_pipeline_validated
    bad = [dataclasses.replace(e, acceptance=0.99) for e in ev]
    assert not P.observed_phase3f_receipt_matches(P.summarize_surfaces(bad, rejected))
