"""Two-row binary32 SU(3) storage (configs with FP32 link algebra, FP64 dS,
accept test, plaquette accumulation and reunitarisation) against FP64.

Bars, stated as the error of the FP32 path against the FP64 path:
  * storage round trip: |U_f32 - U| <= 2e-7 per entry (binary32 rounding);
  * one sweep from the same field and streams: >= 98% of links within 1e-5
    of the FP64 result (accept decisions may flip where u lies within the
    ~1e-6 dS error of exp(-dS));
  * plaquette of the same field: <= 1e-6 absolute;
  * equilibrium plaquette (64 chains of 4^4, beta 6.0): within 4 combined
    standard errors of the FP64 sampler's.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rough(oracle, ext, seed, sweeps=3):
    links = oracle.su3_identity(ext, lift_cap=True)
    for s in range(sweeps):
        oracle.su3_cb_sweep(ext, links, 0.0, 1.0, seed, s)
    return links


def test_two_row_round_trip_and_plaquette(oracle):
    import ymgpu
    ext = [4, 4, 4, 6]
    links = rough(oracle, ext, 2)
    with ymgpu.Ensemble([ext], 6.0, 0, precision=ymgpu.F32_TWO_ROW) as ens:
        ens.upload(0, links)
        back = ens.download(0)
        plaq = ens.average_plaquette()[0]
    assert np.max(np.abs(back - links)) <= 2e-7
    assert abs(plaq - oracle.su3_average_plaquette(ext, links)) <= 1e-6


def test_one_sweep_against_fp64(oracle):
    import ymgpu
    ext = [4, 4, 4, 4]
    links = rough(oracle, ext, 4)
    seed = oracle.derive_su3_chain_seed(0x3C00198212230101, 9)
    with ymgpu.Ensemble([ext], 6.0, seed, precision=ymgpu.F32_TWO_ROW) as e32, \
            ymgpu.Ensemble([ext], 6.0, seed) as e64:
        e32.upload(0, links)
        e64.upload(0, links)
        e32.metropolis_sweeps(0.3, 1)
        e64.metropolis_sweeps(0.3, 1)
        a = e32.download(0)
        b = e64.download(0)
        p32, a32 = e32.accounting()
        p64, a64 = e64.accounting()
    per_link = np.abs(a - b).reshape(len(a), -1).max(1)
    assert np.mean(per_link <= 1e-5) >= 0.98
    assert p32[0] == p64[0] and abs(int(a32[0]) - int(a64[0])) <= 0.01 * int(p64[0])


def test_reunitarize_and_convert(oracle):
    import ymgpu
    ext = [4, 4, 4, 4]
    with ymgpu.Ensemble([ext], 6.0, 17, precision=ymgpu.F32_TWO_ROW) as e32:
        e32.hot_start()
        e32.metropolis_sweeps(0.5, 40)
        e32.reunitarize()
        e64 = e32.like(precision=ymgpu.F64)
        e32.convert_to(e64)
        u, d = e64.max_residuals()
        w = e64.wilson_loops(1, 1)[0]
        p64 = e64.average_plaquette()[0]
        p32 = e32.average_plaquette()[0]
        from ymgpu.errors import YmError
        with pytest.raises(YmError) as err:
            e32.max_residuals()
        assert err.value.variant == "UnsupportedPrecision"
        e64.close()
    assert u[0] <= 1e-6 and d[0] <= 1e-6
    assert abs(p64 - p32) <= 1e-14
    assert abs(np.mean(w[:, 0, 0]) - p64) <= 1e-12


def test_equilibrium_plaquette_fp32_vs_fp64():
    import ymgpu
    from ymgpu.su3_ensemble import derive_su3_chain_seed
    nch = 64
    seeds = [derive_su3_chain_seed(0x2C02198105010002, i) for i in range(nch)]
    res = {}
    for name, prec in (("f32", ymgpu.F32_TWO_ROW), ("f64", ymgpu.F64)):
        with ymgpu.Ensemble([[4, 4, 4, 4]] * nch, 6.0, seeds, precision=prec) as ens:
            ens.metropolis_sweeps(0.35, 200)
            series = np.zeros((nch, 100))
            for m in range(100):
                ens.metropolis_sweeps(0.35, 2)
                series[:, m] = ens.average_plaquette()
        means = series.mean(1)
        res[name] = (means.mean(), means.std(ddof=1) / np.sqrt(nch))
    d = abs(res["f32"][0] - res["f64"][0])
    assert d <= 4.0 * np.hypot(res["f32"][1], res["f64"][1]), res


def test_two_row_sweeps_stay_unitary():
    """Wide proposals for many sweeps: the per-sweep reunitarisation keeps the
    two-row links on the group (without it the deviation grows geometrically
    and reaches non-finite values within a few hundred sweeps)."""
    import ymgpu
    with ymgpu.Ensemble([[4, 4, 4, 6]] * 8, 6.0, list(range(8)),
                        precision=ymgpu.F32_TWO_ROW) as e32:
        e32.hot_start()
        e32.metropolis_sweeps(1.0, 400)
        p = e32.average_plaquette()
        e64 = e32.like(precision=ymgpu.F64)
        e32.convert_to(e64)
        u, d = e64.max_residuals()
        e64.close()
    assert np.all(np.isfinite(p)) and np.all(p > 0.4)
    assert np.all(u <= 1e-6) and np.all(d <= 1e-6)
