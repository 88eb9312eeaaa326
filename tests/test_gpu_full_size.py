"""Parity at the workloads' full sizes, through properties that do not need
the oracle to sweep the whole lattice.

* 32^4 and 24^3 x 48 FP64 (the FP64 and FP32 sweep workloads): after one GPU
  sweep, sampled links are recomputed by the oracle from the neighbourhood
  each one saw when its sub-sweep ran — staple links of earlier checkerboard
  sub-sweeps (parity 0 then 1, direction 0..3) at their post-sweep values,
  later ones at their pre-sweep values — and must equal the GPU's links bit
  for bit; the lattice plaquette matches the oracle's sequential sum to
  1e-12 relative and the links stay in SU(3) to 1e-12.
* 32^4 and 24^3 x 48 two-row FP32: one sweep from the same field, seed and
  sweep index as the FP64 sweep stays within the FP32 path's stated error of
  it.
* SU(2) 10^4 at beta 2.3 (the heat-bath workload): the GPU sweep equals the
  oracle's checkerboard sweep (overrelaxation bitwise, heat-bath to 1e-12).
* 64 chains of 4^4 (the batched-chain workload): chains across the batch
  equal the oracle bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASTER = 0x2C02198105010002


def _neighbour(ext, x, d, step):
    y = list(x)
    y[d] = (y[d] + step) % ext[d]
    return tuple(y)


def _lex(ext, x):
    return ((x[0] * ext[1] + x[1]) * ext[2] + x[2]) * ext[3] + x[3]


def _coords(ext, lex):
    x3 = lex % ext[3]
    r = lex // ext[3]
    x2 = r % ext[2]
    r //= ext[2]
    return (r // ext[1], r % ext[1], x2, x3)


def _order(x, mu):
    """Position of link (x, mu) in the sweep: parity 0 then 1, mu 0..3."""
    return (sum(x) & 1) * 4 + mu


def _staple_links(ext, x, mu):
    out = []
    for nu in range(4):
        if nu == mu:
            continue
        xpm = _neighbour(ext, x, mu, +1)
        xpn = _neighbour(ext, x, nu, +1)
        xmn = _neighbour(ext, x, nu, -1)
        xmnpm = _neighbour(ext, xmn, mu, +1)
        out += [(xpm, nu), (xpn, mu), (x, nu), (xmnpm, nu), (xmn, mu), (xmn, nu)]
    return out


def _check_sampled_links(oracle, ext, before, after, seed, sweep, angle, uniform, n_samples, rng):
    """Recompute n_samples links of `after` from `before`/`after` with the
    oracle and compare bitwise."""
    n_sites = int(np.prod(ext))
    lexes = rng.integers(0, n_sites, n_samples)
    mus = rng.integers(0, 4, n_samples)
    work = before          # patched in place, restored after each sample
    for lex, mu in zip(lexes.tolist(), mus.tolist()):
        x = _coords(ext, lex)
        k = _order(x, mu)
        patched = []
        for (y, nu) in _staple_links(ext, x, mu):
            if _order(y, nu) < k:
                idx = _lex(ext, y) * 4 + nu
                patched.append((idx, work[idx].copy()))
                work[idx] = after[idx]
        a = oracle.su3_staple(ext, work, x, mu)
        for idx, old in reversed(patched):
            work[idx] = old
        key = oracle.cb_link_key(seed, sweep, lex, mu)
        u, _ = oracle.su3_visit(work[lex * 4 + mu], a, 6.0, angle, key, uniform)
        assert np.array_equal(u, after[lex * 4 + mu]), (x, mu)


@pytest.mark.parametrize("ext,uniform", [([32, 32, 32, 32], False), ([32, 32, 32, 32], True),
                                         ([24, 24, 24, 48], False)])
def test_full_size_sweep_sampled_links_bitwise(oracle, ext, uniform):
    import ymgpu
    seed = oracle.derive_su3_chain_seed(MASTER, 2)
    with ymgpu.Ensemble([ext], 6.0, seed, lift_reference_caps=True) as ens:
        ens.hot_start()
        ens.metropolis_sweeps(1.0, 3, "uniform")
        before = ens.download(0)
        sweep = ens.sweep_index
        ens.metropolis_sweeps(0.3, 1, "uniform" if uniform else "ordered")
        after = ens.download(0)
        plaq = ens.average_plaquette()[0]
        ures, dres = ens.max_residuals()
    assert not np.array_equal(before, after)
    _check_sampled_links(oracle, ext, before, after, seed, sweep, 0.3, uniform, 1500,
                         np.random.default_rng(7 + int(uniform)))
    ref = oracle.su3_average_plaquette(ext, after)
    assert abs(plaq - ref) <= 1e-12 * abs(ref)
    assert ures[0] <= 1e-12 and dres[0] <= 1e-12


@pytest.mark.parametrize("ext", [[32, 32, 32, 32], [24, 24, 24, 48]])
def test_full_size_fp32_sweep_error_against_fp64(oracle, ext):
    """The two-row binary32 sweep at 32^4 and 24^3 x 48, from the same field,
    seed and sweep index as the FP64 sweep (bitwise the oracle's, above):
    >= 98% of links within 1e-5 of the FP64 result (a decision may flip where
    the uniform lies within the ~1e-6 dS error of exp(-dS)), plaquettes
    within 1e-6."""
    import ymgpu
    seed = oracle.derive_su3_chain_seed(MASTER, 5)
    with ymgpu.Ensemble([ext], 6.0, seed, lift_reference_caps=True) as e64, \
            ymgpu.Ensemble([ext], 6.0, seed, precision=ymgpu.F32_TWO_ROW,
                           lift_reference_caps=True) as e32:
        e64.hot_start()
        e64.metropolis_sweeps(1.0, 3, "uniform")
        e32.upload(0, e64.download(0))
        e32.sweep_index = e64.sweep_index
        e64.metropolis_sweeps(0.3, 1)
        e32.metropolis_sweeps(0.3, 1)
        a = e64.download(0)
        b = e32.download(0)
        p64 = e64.average_plaquette()[0]
        p32 = e32.average_plaquette()[0]
    per_link = np.abs(a - b).reshape(len(a), -1).max(1)
    assert np.mean(per_link <= 1e-5) >= 0.98
    assert abs(p64 - p32) <= 1e-6


def test_su2_10x4_sweep_equals_oracle(oracle):
    import ctypes as C
    import ymgpu
    ext = [10, 10, 10, 10]
    seed = oracle.derive_chain_seed(0x2B0020121116_0101, 0)
    start = oracle.su2_identity(ext)
    for s in range(2):
        oracle.su2_cb_sweep(ext, start, 1.0, 99, s, 1, 100000)
    with ymgpu.Ensemble([ext], 2.3, seed, group=ymgpu.SU2) as ens:
        ens.upload(0, start)
        ens.overrelaxation_sweeps(1)
        gpu_or = ens.download(0)
    with ymgpu.Ensemble([ext], 2.3, seed, group=ymgpu.SU2) as ens:
        ens.upload(0, start)
        ens.markov_sweeps(1, overrelaxation_sweeps=3, max_attempts_per_link=10000,
                          sampler="reference")
        gpu = ens.download(0)
    L = oracle.lib()
    L.or_su2_cb_overrelax.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    cpu_or = start.copy()
    assert L.or_su2_cb_overrelax((C.c_int64 * 4)(*ext),
                                 cpu_or.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert np.array_equal(gpu_or, cpu_or)
    cpu = start.copy()
    oracle.su2_cb_sweep(ext, cpu, 2.3, seed, 0, 3, 10000)
    assert np.max(np.abs(gpu - cpu)) <= 1e-12


def test_64_chains_of_4x4_equal_oracle(oracle):
    import ymgpu
    ext = [4, 4, 4, 4]
    seeds = [oracle.derive_su3_chain_seed(MASTER, i) for i in range(64)]
    with ymgpu.Ensemble([ext] * 64, 6.0, seeds) as ens:
        ens.metropolis_sweeps(0.3, 3, "uniform")
        got = {i: ens.download(i) for i in (0, 31, 63)}
        prop, acc = ens.accounting()
    for i, links in got.items():
        cpu = oracle.su3_identity(ext)
        na = 0
        for s in range(3):
            na += oracle.su3_cb_sweep(ext, cpu, 6.0, 0.3, seeds[i], s, True)[1]
        assert np.array_equal(links, cpu), i
        assert int(acc[i]) == na
