"""Chain-resident sweeps (small chains kept in one CTA's shared memory for
many sweeps per launch) against the oracle and against the tiled launches.
Bars: links, accept counts and the sweep counter bitwise equal to the
oracle's restatement of the checkerboard order; measured plaquette series
bitwise equal to the tiled path's (the same per-site sums and reduction
tree)."""
import numpy as np
import pytest

from test_gpu_su3 import MASTER, rough_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["ordered", "uniform"])
def test_resident_sweeps_bitwise_equal_oracle(oracle, mode):
    import ymgpu
    exts = [[4, 4, 4, 4], [2, 4, 4, 6], [2, 2, 4, 4]]
    betas = [6.0, 5.7, 0.0]
    seeds = [oracle.derive_su3_chain_seed(MASTER, 40 + i) for i in range(3)]
    starts = [rough_config(oracle, e, 50 + i, 2) for i, e in enumerate(exts)]
    with ymgpu.Ensemble(exts, betas, seeds) as ens:
        ens.sweep_path = "resident"
        for i, s in enumerate(starts):
            ens.upload(i, s)
        ens.sweep_index = 5
        ens.metropolis_sweeps(0.3, 3, mode)
        gpu = [ens.download(i) for i in range(3)]
        prop, acc = ens.accounting()
        assert ens.sweep_index == 8 and ens.sweep_path == "resident"
    for i, e in enumerate(exts):
        cpu = starts[i].copy()
        na = 0
        for s in range(5, 8):
            _, a = oracle.su3_cb_sweep(e, cpu, betas[i], 0.3, seeds[i], s, mode == "uniform")
            na += a
        assert np.array_equal(gpu[i], cpu), f"chain {i}"
        assert int(acc[i]) == na and int(prop[i]) == 3 * 32 * int(np.prod(e))


def test_resident_measured_series_equals_tiled():
    import ymgpu
    from ymgpu.su3_ensemble import derive_su3_chain_seed
    seeds = [derive_su3_chain_seed(9, i) for i in range(12)]
    exts = [[4, 4, 4, 4]] * 10 + [[2, 4, 4, 6]] * 2
    with ymgpu.Ensemble(exts, 6.0, seeds) as a, ymgpu.Ensemble(exts, 6.0, seeds) as b:
        a.sweep_path = "resident"
        b.sweep_path = "tiled"
        for e in (a, b):
            e.hot_start()
        sa = a.measured_sweeps(0.3, 25, 2, "uniform")
        sb = b.measured_sweeps(0.3, 25, 2, "uniform")
        assert np.array_equal(sa, sb)
        assert np.array_equal(a.average_plaquette(), b.average_plaquette())
        assert np.array_equal(a.accounting()[1], b.accounting()[1])
        assert a.sweep_index == b.sweep_index == 50
        for c in (0, 11):
            assert np.array_equal(a.download(c), b.download(c))


def test_auto_path_decides_and_matches_tiled():
    import ymgpu
    from ymgpu.su3_ensemble import derive_su3_chain_seed
    seeds = [derive_su3_chain_seed(3, i) for i in range(64)]
    with ymgpu.Ensemble([[4, 4, 4, 4]] * 64, 6.0, seeds) as a, \
            ymgpu.Ensemble([[4, 4, 4, 4]] * 64, 6.0, seeds) as b:
        b.sweep_path = "tiled"
        assert a.sweep_path == "auto"
        a.metropolis_sweeps(0.3, 40, "ordered")
        b.metropolis_sweeps(0.3, 40, "ordered")
        assert a.sweep_path in ("tiled", "resident")
        sa = a.measured_sweeps(0.3, 10, 1, "ordered")
        sb = b.measured_sweeps(0.3, 10, 1, "ordered")
        assert np.array_equal(sa, sb)
        assert np.array_equal(a.download(63), b.download(63))


def test_resident_rejects_large_or_two_row():
    import ymgpu
    from ymgpu.errors import YmError
    with ymgpu.Ensemble([[8, 8, 8, 8]], 6.0, 1) as big, \
            ymgpu.Ensemble([[4, 4, 4, 4]], 6.0, 1, precision=ymgpu.F32_TWO_ROW) as f32:
        for e in (big, f32):
            with pytest.raises(YmError) as err:
                e.sweep_path = "resident"
            assert err.value.variant == "InvalidArgument"
        big.metropolis_sweeps(0.3, 9)          # auto stays tiled: the chain does not fit
        assert big.sweep_path == "auto"
