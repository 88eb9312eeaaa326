"""The fast form of the SU(3) FP64 sweep (ym_ensemble_set_fast_sweeps).

The fast form runs the reference's algorithm, streams and binary64 links
with fused multiply-adds and Horner rotations, so it is held to a distance
from the reference's bits rather than to them:

  * against the oracle's checkerboard sweeps from the same start, seed and
    sweep index: every link entry within 1e-14, the same accept count;
  * against the exact GPU sweep over 10 sweeps of a 16^4 Haar start: every
    entry within 1e-13 (measured 3.2e-15), the same accept count;
  * unitarity and determinant residuals of the swept links <= 1e-14;
  * the flag's API: default off, binary64 SU(3) only, no chain-resident
    path while on, and captured sweep graphs rebuilt when it changes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASTER = 0x3C00198212230101


def _rough(oracle, ext, seed, sweeps=3):
    links = oracle.su3_identity(ext, lift_cap=True)
    for s in range(sweeps):
        oracle.su3_cb_sweep(ext, links, 0.0, 1.0, seed, s)
    return links


@pytest.mark.parametrize("uniform", [False, True])
@pytest.mark.parametrize("angle", [0.3, 1.0])
def test_fast_sweeps_within_1e14_of_oracle(oracle, uniform, angle):
    import ymgpu
    ext = [4, 4, 4, 4]
    start = _rough(oracle, ext, 5)
    seed = oracle.derive_su3_chain_seed(MASTER, 7)
    with ymgpu.Ensemble([ext], 6.0, seed) as ens:
        ens.fast_sweeps = True
        ens.upload(0, start)
        ens.sweep_index = 11
        ens.metropolis_sweeps(angle, 3, "uniform" if uniform else "ordered")
        gpu = ens.download(0)
        prop, acc = ens.accounting()
    cpu = start.copy()
    np_, na = 0, 0
    for s in range(11, 14):
        p, a = oracle.su3_cb_sweep(ext, cpu, 6.0, angle, seed, s, uniform)
        np_ += p
        na += a
    assert int(prop[0]) == np_ and int(acc[0]) == na
    diff = np.max(np.abs(gpu - cpu))
    assert diff <= 1e-14, diff
    assert not np.array_equal(gpu, cpu)       # the fast form really ran


def test_fast_sweeps_track_exact_sweeps_at_16x4():
    import ymgpu
    ext = [16, 16, 16, 16]
    with ymgpu.Ensemble([ext], 6.0, 0x77, lift_reference_caps=True) as ex, \
            ymgpu.Ensemble([ext], 6.0, 0x77, lift_reference_caps=True) as fa:
        fa.fast_sweeps = True
        for e in (ex, fa):
            e.hot_start()
            e.metropolis_sweeps(0.3, 10, "ordered")
        a, b = ex.download(0), fa.download(0)
        assert np.array_equal(ex.accounting()[1], fa.accounting()[1])
        diff = np.max(np.abs(a - b))
        assert 0.0 < diff <= 1e-13, diff
        u, d = fa.max_residuals()
        assert u.max() <= 1e-14 and d.max() <= 1e-14, (u, d)
        assert abs(ex.average_plaquette()[0] - fa.average_plaquette()[0]) <= 1e-13


def test_fast_flag_api_and_graph_rebuild():
    import ymgpu
    from ymgpu.ensemble import F32_TWO_ROW
    from ymgpu.errors import YmError
    ext = [8, 8, 8, 8]
    with ymgpu.Ensemble([ext], 6.0, 0x99) as a, ymgpu.Ensemble([ext], 6.0, 0x99) as b:
        assert a.fast_sweeps is False
        for e in (a, b):
            e.hot_start()
            e.metropolis_sweeps(0.3, 16, "ordered")      # two captured 8-sweep batches
        a.fast_sweeps = True                              # the captured graph must go
        a.metropolis_sweeps(0.3, 16, "ordered")
        b.metropolis_sweeps(0.3, 16, "ordered")
        la, lb = a.download(0), b.download(0)
        assert not np.array_equal(la, lb)
        assert np.max(np.abs(la - lb)) <= 1e-13
        a.fast_sweeps = False
        assert a.fast_sweeps is False
    with ymgpu.Ensemble([[4, 4, 4, 4]] * 8, 6.0, list(range(8))) as small:
        small.fast_sweeps = True
        with pytest.raises(YmError):
            small.sweep_path = "resident"                 # fast sweeps are tiled only
        small.fast_sweeps = False
        small.sweep_path = "resident"
        assert ymgpu.lib().ym_ensemble_set_fast_sweeps(small.handle, 2) != 0   # only 0 or 1
    with ymgpu.Ensemble([ext], 6.0, 0x99, precision=F32_TWO_ROW) as f:
        with pytest.raises(YmError):
            f.fast_sweeps = True
