"""The phase-3F production campaign end to end with its sixteen chains on
the device (glueball_scalar_production.rs:640-720): schedule accounting,
acceptance and residual gates, the six (transformation, operator)
surfaces with correlators replaying the frozen estimator, and the summary's
gates applied to the fits."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_production_campaign_on_device(oracle):
    from ymgpu import production as P
    s = P.run_production_scalar_analysis()
    assert len(s.chain_evidence) == P.CHAIN_COUNT
    for e in s.chain_evidence:
        assert e.proposals == P.EXPECTED_PROPOSALS_PER_CHAIN
        assert P.MIN_ACCEPTANCE <= e.acceptance <= P.MAX_ACCEPTANCE
        assert e.unitarity_residual <= P.LINK_RESIDUAL_LIMIT and e.determinant_residual <= P.LINK_RESIDUAL_LIMIT
    assert s.sampler_diagnostics_passed
    assert [(r.outcome.transformation, r.outcome.operator) for r in s.surfaces] == \
        [(t, o) for t, o, _ in P.OBSERVED_SURFACE_OUTCOMES]
    for r in s.surfaces:
        assert r.outcome.succeeded() != (r.outcome.error_code is not None)
        assert len(r.correlator.jackknife) == P.CHAIN_COUNT
        assert r.correlator.full.shape == (P.EXTENTS[3],)
    # the reference's own run (glueball-scalar-production-phase3f-v1,
    # "observed-negative-production-receipt") rejected all six surfaces on
    # the effective mass; the device chains reproduce that receipt
    assert P.observed_phase3f_receipt_matches(s)
    # the summary's gates are consistent with the surfaces it was given
    again = P.summarize_surfaces(s.chain_evidence, s.surfaces)
    assert again.scalar_pipeline_validated == s.scalar_pipeline_validated
    assert again.primary_window_successes == s.primary_window_successes


def test_recovery_campaigns_reproduce_the_recorded_receipts():
    """Phases 3G and 3H (glueball_scalar_recovery_receipt.rs,
    glueball_scalar_geometry_recovery_receipt.rs) recorded all surfaces
    rejected on the effective mass; phase 3I has no recorded outcome and
    runs to a complete summary (2.4e8 proposals)."""
    from ymgpu import production as P
    for name in ("phase3g", "phase3h"):
        c = P.CAMPAIGNS[name]
        s = P.run_campaign(c)
        assert P.observed_receipt_matches(s, c), name
    c = P.CAMPAIGNS["phase3i"]
    s = P.run_campaign(c)
    assert c.expected_proposals_per_chain * c.chain_count == 240_648_192
    assert s.sampler_diagnostics_passed and len(s.surfaces) == 8
    assert [(r.outcome.transformation, r.outcome.operator) for r in s.surfaces] == \
        [(t, o) for t, _, _ in c.transformations for o in P.OPERATORS]
