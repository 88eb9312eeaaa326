"""The run_chain cadence's plaquette taken from the sweep (ym_su3_measured_sweeps,
ym_su3_measured_run).

For binary64 handles with ordered hits whose chains are too large for the
chain-resident kernel, sub-sweeps (parity 1, direction mu = 1, 2, 3) of each
measured sweep sum (1/3) Re Tr(U' A_p) of their links, A_p the staple terms
of the directions below mu: the plaquettes of planes (0,1); (0,2), (1,2);
(0,3), (1,3), (2,3).  No plaquette kernel runs.  The sweeps themselves are
unchanged, so:

  * the links, accept counts and sweep index after measured sweeps are
    bitwise those of the same sweeps launched directly;
  * every plaquette of the series is within 1e-12 relative of
    ym_average_plaquette after the same sweep (a different summation
    order), and of the oracle's plaquette after the oracle's sweeps;
  * uneven chains in one handle each get their own plaquette.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASTER = 0x3C00198212230101


def _rough(oracle, ext, seed, sweeps=2):
    links = oracle.su3_identity(ext, lift_cap=True)
    for s in range(sweeps):
        oracle.su3_cb_sweep(ext, links, 0.0, 1.0, seed, s)
    return links


@pytest.mark.parametrize("per", [1, 2])
def test_measured_series_matches_direct_launches(oracle, per):
    import ymgpu
    exts = [[8, 8, 8, 8], [6, 6, 6, 8], [8, 4, 4, 10]]
    seeds = [oracle.derive_su3_chain_seed(MASTER, i) for i in range(3)]
    starts = [_rough(oracle, x, 11 + i) for i, x in enumerate(exts)]
    with ymgpu.Ensemble(exts, 6.0, seeds) as a, ymgpu.Ensemble(exts, 6.0, seeds) as b:
        for e in (a, b):
            for i, s in enumerate(starts):
                e.upload(i, s)
            e.sweep_index = 3
        series = a.measured_sweeps(0.3, 6, per, "ordered")
        direct = []
        for _ in range(6):
            b.metropolis_sweeps(0.3, per)
            direct.append(b.average_plaquette())
        direct = np.array(direct)
        assert np.all(np.abs(series - direct) <= 1e-12 * np.abs(direct))
        for i in range(3):
            assert np.array_equal(a.download(i), b.download(i))
        assert np.array_equal(a.accounting()[1], b.accounting()[1])
        assert a.sweep_index == b.sweep_index == 3 + 6 * per


def test_measured_series_matches_oracle(oracle):
    import ymgpu
    ext = [8, 8, 8, 8]
    start = _rough(oracle, ext, 5)
    seed = oracle.derive_su3_chain_seed(MASTER, 9)
    with ymgpu.Ensemble([ext], 6.0, seed) as e:
        e.upload(0, start)
        e.sweep_index = 7
        series = e.measured_sweeps(0.3, 3, 1, "ordered")[:, 0]
        gpu_links = e.download(0)
    cpu = start.copy()
    for k, s in enumerate((7, 8, 9)):
        oracle.su3_cb_sweep(ext, cpu, 6.0, 0.3, seed, s)
        want = oracle.su3_average_plaquette(ext, cpu)
        assert abs(series[k] - want) <= 1e-12 * abs(want)
    assert np.array_equal(gpu_links, cpu)


def test_measured_run_plaquettes_match_measured_sweeps(oracle):
    import ymgpu
    ext = [8, 8, 8, 8]
    start = _rough(oracle, ext, 2)
    with ymgpu.Ensemble([ext], 6.0, 21) as a, ymgpu.Ensemble([ext], 6.0, 21) as b:
        for e in (a, b):
            e.upload(0, start)
        plaq, _, _ = a.measured_run(0.3, 2, 3, 4, 3, 3, "ordered")
        ref = b.measured_sweeps(0.3, 6, 1, "ordered")
        assert np.array_equal(plaq, ref)
        assert np.array_equal(a.download(0), b.download(0))
