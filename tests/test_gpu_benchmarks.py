"""The frozen published-baseline harnesses run end to end on device chains
(su2_benchmark.rs, su3_benchmark.rs, su3_confirmation.rs): every structural
gate passes and the published plaquette envelopes are reproduced."""
import pytest

pytestmark = pytest.mark.gpu


def test_su2_published_baseline_on_device():
    from ymgpu import benchmarks as B
    s = B.run_su2_benchmark()
    assert B.su2.SOURCE_ENVELOPE_MIN <= s.pooled_mean <= B.su2.SOURCE_ENVELOPE_MAX
    assert s.max_link_unit_residual <= B.su2.MAX_LINK_UNIT_RESIDUAL
    assert s.phase2_graduation_gate_satisfied, s


def test_su3_published_baseline_and_confirmation_on_device():
    from ymgpu import benchmarks as B
    s = B.run_su3_benchmark()
    assert all(B.su3.MIN_METROPOLIS_ACCEPTANCE <= a <= B.su3.MAX_METROPOLIS_ACCEPTANCE
               for a in s.chain_acceptances)
    assert s.published_su3_baseline_reproduced, s
    c = B.run_su3_confirmation()
    assert c.published_su3_baseline_reproduced, c
