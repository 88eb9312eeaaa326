"""The variational cross-correlator from device operator samples
(glueball_scalar_variational.rs:628-744 with the A1++ basis evaluated by the
engine on every chain) against the oracle, its diagonal replay of the
single-operator correlators, gauge invariance (glueball_scalar_variational.rs:1040-1058)
and the downstream effective mass / GEVP chain on the same configurations."""
import numpy as np
import pytest

import analysis_oracle as AO

pytestmark = pytest.mark.gpu


def rough(oracle, ext, seed, sweeps=2):
    links = oracle.su3_identity(ext, lift_cap=True)
    for s in range(sweeps):
        oracle.su3_cb_sweep(ext, links, 0.0, 0.6, seed, s)
    return links


def test_variational_correlator_from_device_samples(oracle):
    import ymgpu
    from ymgpu import analysis as A
    from ymgpu import glueball as G
    ext = [4, 4, 4, 6]
    n = 5
    lats = [rough(oracle, ext, 100 + k) for k in range(n)]
    with ymgpu.Ensemble([ext] * n, 6.0, list(range(n))) as ens:
        for k, lat in enumerate(lats):
            ens.upload(k, lat)
        var = A.scalar_variational_connected_correlator(ens)
        diag = G.scalar_connected_correlators(ens)
        p, r = G.operator_samples(ens)
    # the operator samples are the oracle's per-slice basis to 1e-12
    for k, lat in enumerate(lats):
        for t in range(ext[3]):
            b = oracle.scalar_a1pp_operator_basis(ext, lat, t)
            assert abs(p[k, t] - b[0]) <= 1e-12 and abs(r[k, t] - b[1]) <= 1e-12
    (v0, v1), mats = AO.variational_correlator_from_samples(p.tolist(), r.tolist())
    assert var.vacuum_means == (v0, v1)
    assert np.array_equal(var.matrices, np.array(mats))
    assert var.configuration_count == n and var.time_extent == ext[3]
    for tau in range(ext[3]):
        assert abs(var.matrices[tau][0][0] - diag.plaquette_connected[tau]) <= A.SYMMETRY_TOLERANCE
        assert abs(var.matrices[tau][1][1] - diag.rectangle_connected[tau]) <= A.SYMMETRY_TOLERANCE
        assert var.matrices[tau][0][1] == var.matrices[tau][1][0]
    # gauge invariance of the whole matrix series
    g = oracle.su3_deterministic_gauge_field(ext)
    with ymgpu.Ensemble([ext] * n, 6.0, list(range(n))) as ens:
        for k, lat in enumerate(lats):
            ens.upload(k, oracle.su3_gauge_transform(ext, lat, g))
        var_g = A.scalar_variational_connected_correlator(ens)
    assert A.max_matrix_series_residual(var.matrices, var_g.matrices) <= A.GAUGE_INVARIANCE_TOLERANCE


def test_analysis_chain_on_device_correlators(oracle):
    """Jackknife replicas of the device plaquette correlator feed the cosh
    effective mass; engine and oracle agree bit for bit on every step."""
    import ymgpu
    from ymgpu import analysis as A
    from ymgpu import glueball as G
    ext = [4, 4, 4, 8]
    n = 6
    with ymgpu.Ensemble([ext] * n, 5.7, [0x77 + k for k in range(n)]) as ens:
        ens.hot_start()
        ens.metropolis_sweeps(0.3, 10, "uniform")
        p, _ = G.operator_samples(ens)
    full = G.connected_from_samples(p)
    jk = G.jackknife_replicas(p)
    lags = [1, 2, 3]
    try:
        ref = AO.cosh_effective_mass_with_jackknife(full, jk, lags)
    except AO.AnalysisError as e:
        from ymgpu.errors import YmError
        with pytest.raises(YmError) as err:
            A.cosh_effective_mass_with_jackknife(full, jk, lags)
        assert err.value.variant == e.variant
        return
    got = A.cosh_effective_mass_with_jackknife(full, jk, lags)
    assert [(q.tau, q.full_estimate, q.jackknife_mean, q.standard_error) for q in got.points] == ref
