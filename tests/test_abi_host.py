"""CPU checks of the C-ABI library: it loads, exports every symbol the
headers declare, and its host-side logic (stream seeds, angle grid,
diagnostics, sampling efficiency) equals the oracle.  No device call."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(ym_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import ymgpu
    L = C.CDLL(ymgpu.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    assert len(declared_symbols()) >= 20


def test_python_mirror_binds_every_symbol():
    from ymgpu import _lib
    bound = set(_lib.SIGNATURES) | set(_lib.U64_FUNCTIONS)
    assert set(declared_symbols()) <= bound, set(declared_symbols()) - bound


def test_status_codes_map_to_reference_variants():
    from ymgpu.errors import CODES, VARIANTS
    assert CODES[38] == "NonFiniteStatistic"
    assert VARIANTS["BetaOutsideReferenceRange"] == 30
    assert VARIANTS["ProposalAngleOutsideReferenceRange"] == 70


def test_seeds_and_angle_grid_match_oracle(oracle):
    from ymgpu import su2_ensemble as S2, su3_ensemble as S3
    rng = np.random.default_rng(0)
    for _ in range(50):
        m, c = int(rng.integers(0, 2**63)), int(rng.integers(0, 1000))
        assert S3.derive_su3_chain_seed(m, c) == oracle.derive_su3_chain_seed(m, c)
        assert S2.derive_chain_seed(m, c) == oracle.derive_chain_seed(m, c)
        raw = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
        assert S3.proposal_angle_from_u64(raw, 0.3) == oracle.proposal_angle_from_u64(raw, 0.3)
        assert S2.splitmix64_at(m, c) == oracle.splitmix_at(m, c)
    from ymgpu.errors import YmError
    with pytest.raises(YmError) as e:
        S3.proposal_angle_from_u64(1, 0.0)
    assert e.value.variant == "ProposalAngleOutsideReferenceRange"


def test_host_diagnostics_equal_oracle(oracle, golden):
    from ymgpu import su2_ensemble as S2
    v = [x for x in golden["su3-ensemble-v1.json"]["vectors"]
         if x["id"] == "frozen-reference-chain-golden-evidence"][0]
    meas = np.array(v["raw_measurements"])
    d, ac = S2.diagnostics(meas, 4)
    od, oac = oracle.diagnostics(meas, 4)
    assert d.mean == od.mean and d.variance == od.variance
    assert d.integrated_autocorrelation_time == od.integrated_autocorrelation_time
    assert d.effective_sample_size == od.effective_sample_size
    assert np.array_equal(ac, oac)


def test_host_sampling_efficiency_vectors(golden):
    from ymgpu import su2_ensemble as S2
    v = golden["sampling-efficiency-v1.json"]
    c = v["cost"]
    e = S2.sampling_efficiency(v["values"], np.log([1, 1, 1, 3]), v["max_lag"], c["setup"],
                               c["thermalization"], c["sampling"])
    w = v["weights_1_1_1_3"]
    assert abs(e.reweighting_efficiency - w["weight_efficiency"]) <= v["tolerance"]
    assert abs(e.total_cost_per_effective_sample_proxy - w["total_cost_per_proxy"]) <= v["tolerance"]


def test_config_validation_fails_closed():
    """su3_ensemble.rs:280-309 error paths through the mirror's validate()."""
    from ymgpu.su3_ensemble import Su3EnsembleConfig, MAX_REFERENCE_SWEEPS
    from ymgpu.errors import YmError
    base = dict(extents=[2, 2, 2, 2], beta=0.0, master_seed=1, chain_id=0,
                thermalization_sweeps=2, measurements=8, sweeps_between_measurements=1,
                proposal_angle=0.35, autocorrelation_max_lag=3)
    for change, variant in [(dict(proposal_angle=0.0), "ProposalAngleOutsideReferenceRange"),
                            (dict(beta=float("nan")), "BetaOutsideReferenceRange"),
                            (dict(sweeps_between_measurements=0), "ZeroMeasurementStride"),
                            (dict(thermalization_sweeps=MAX_REFERENCE_SWEEPS),
                             "ScheduleOutsideReferenceRange"),
                            (dict(extents=[32, 32, 32, 32]), "LatticeOutsideReferenceRange")]:
        cfg = Su3EnsembleConfig(**{**base, **change})
        with pytest.raises(YmError) as e:
            cfg.validate()
        assert e.value.variant == variant
    Su3EnsembleConfig(**{**base, "extents": [32, 32, 32, 32]}).validate(lift_reference_caps=True)


def test_jackknife_replicas_every_replica_and_failures(oracle):
    """Every delete-one replica (computed on the host's threads from shared
    products) equals the one-replica function bit for bit, and a rejected
    input returns the status the one-at-a-time loop returns."""
    from ymgpu import glueball as G
    from ymgpu.errors import YmError
    rng = np.random.default_rng(11)
    s = rng.normal(0.9, 0.02, size=(300, 12))
    reps = G.jackknife_replicas(s)
    for k in range(300):
        assert np.array_equal(reps[k], G.connected_from_samples(s, k)), k
    for k in (0, 149, 299):
        assert np.array_equal(reps[k], oracle.connected_from_samples(s, k))
    bad = s.copy()
    bad[5, 3] = np.nan
    with pytest.raises(YmError) as e:
        G.jackknife_replicas(bad)
    assert e.value.variant == "NonFiniteStatistic"
    with pytest.raises(YmError) as e:
        G.jackknife_replicas(s[:1])
    assert e.value.variant == "EmptyConfigurationSet"


def test_host_correlators_equal_oracle(oracle, golden):
    """Connected correlators, delete-one jackknife and covariance: the
    library's host FP64 code equals the oracle bit for bit."""
    from ymgpu import glueball as G
    rng = np.random.default_rng(5)
    s = rng.normal(0.9, 0.02, size=(20, 10))
    vac, raw, con = G.periodic_connected_estimator(s)
    ov, oraw, ocon = oracle.periodic_connected_estimator(s)
    assert vac == ov and np.array_equal(raw, oraw) and np.array_equal(con, ocon)
    reps = G.jackknife_replicas(s)
    for k in (0, 7, 19):
        assert np.array_equal(reps[k], oracle.connected_from_samples(s, k))
    assert np.array_equal(G.connected_from_samples(s), oracle.connected_from_samples(s))
    assert np.array_equal(G.jackknife_covariance(reps, 1, 4), oracle.jackknife_covariance(reps, 1, 4))
    from ymgpu.errors import YmError
    with pytest.raises(YmError) as e:
        G.jackknife_covariance(reps[:3], 1, 4)
    assert e.value.variant == "InsufficientReplicatesForCovariance"
    with pytest.raises(YmError) as e:
        G.connected_from_samples(s, 20)
    assert e.value.variant == "ConfigurationShapeMismatch"
    # the reference's analytic fixture (glueball_correlators.rs:24-33)
    v = [x for x in golden["glueball-connected-correlator-phase3c-v1.json"]["vectors"]
         if x["id"] == "shifted-defect-analytic-correlators"][0]
    p = np.full((4, 4), 79.0 / 81.0)
    for c in range(4):
        p[c, c] = 1.0 - 2.0 / 81.0 + 1.0 / 81.0   # one defect plaquette pair in slice c
    pv, praw, pcon = G.periodic_connected_estimator(
        np.array([[0.9753086419753086] * 4] * 4))
    assert pv == 0.9753086419753086 and np.allclose(pcon, 0.0, atol=1e-15)
