"""The Haar hot start (ym_ensemble_hot_start) pinned by its moments.

The reference always starts cold (su3_ensemble.rs:412), so nothing of the
reference pins the hot start; these tests pin it by what Haar measure on
SU(3) implies for the links it draws, over 4 x 16^4 = 1,048,576 links:

  <Re Tr U> = <Im Tr U> = 0      (Var Re Tr U = Var Im Tr U = 1/2)
  <|Tr U|^2> = 1                 (Var = <|Tr U|^4> - 1 = 1)
  <(Tr U)^3> = 1                 (SU(3), not U(3), where it is 0;
                                  <|Tr U|^6> = 6 bounds its variance)
  <plaquette> = 0                ((1/3) Re Tr of a product of independent
                                  Haar links; variance 1/18 per plaquette,
                                  plaquettes pairwise uncorrelated)

each within 5 standard errors of the sampling error, plus the unitarity and
determinant residuals of the stored links (1e-14 in binary64; binary32
two-row storage rounds to ~6e-8 per entry, so 1e-6 there).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXT = [16, 16, 16, 16]
CHAINS = 4


def _moments(links):
    tr = np.einsum("nii->n", links)
    n = tr.size
    out = {
        "re": (tr.real.mean(), np.sqrt(0.5 / n)),
        "im": (tr.imag.mean(), np.sqrt(0.5 / n)),
        "abs2": (np.mean(np.abs(tr) ** 2) - 1.0, np.sqrt(1.0 / n)),
        "cube_re": (np.mean((tr ** 3).real) - 1.0, np.sqrt(6.0 / n)),
        "cube_im": (np.mean((tr ** 3).imag), np.sqrt(6.0 / n)),
    }
    return out


def _check(ens):
    import ymgpu  # noqa: F401
    links = np.concatenate([ens.download(c) for c in range(ens.n_chains)])
    assert links.shape[0] == CHAINS * 4 * int(np.prod(EXT))
    for name, (dev, se) in _moments(links).items():
        assert abs(dev) <= 5.0 * se, (name, dev, se)
    plaq = ens.average_plaquette()
    n_plaq = 6 * int(np.prod(EXT)) * CHAINS
    assert abs(plaq.mean()) <= 5.0 * np.sqrt(1.0 / 18.0 / n_plaq), plaq
    # Different seeds give different fields; the same seed the same field.
    assert not np.array_equal(links[:16], links[4 * int(np.prod(EXT)):][:16])


def _seeds():
    import oracle as O
    return [O.derive_su3_chain_seed(0x5EED_0000_0000_0018, c) for c in range(CHAINS)]


def test_hot_start_f64_is_haar(oracle):
    import ymgpu
    with ymgpu.Ensemble([EXT] * CHAINS, 6.0, _seeds()) as ens:
        ens.hot_start()
        _check(ens)
        u, d = ens.max_residuals()
        assert u.max() <= 1e-14 and d.max() <= 1e-14, (u, d)
        first = ens.download(0)
        ens.hot_start()                     # the stream is keyed by seed and link: repeatable
        assert np.array_equal(first, ens.download(0))


def test_hot_start_f32_two_row_is_haar(oracle):
    import ymgpu
    from ymgpu.ensemble import F32_TWO_ROW
    with ymgpu.Ensemble([EXT] * CHAINS, 6.0, _seeds(), precision=F32_TWO_ROW) as ens, \
            ymgpu.Ensemble([EXT] * CHAINS, 6.0, _seeds()) as f64:
        ens.hot_start()
        ens.convert_to(f64)                 # binary64 image of the stored two rows
        _check(f64)
        u, d = f64.max_residuals()
        assert u.max() <= 1e-6 and d.max() <= 1e-6, (u, d)
