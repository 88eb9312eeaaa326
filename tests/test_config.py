"""Canonical configuration text (include/ym_config.h) against the reference's
rules (lib.rs:587-694 and its tests lib.rs:1042-1083) and a Python
restatement of the format.  Host code only: no GPU."""
import struct

import numpy as np
import pytest

import config_oracle as CO
from ymgpu import config as K
from ymgpu.errors import YmError


def variant_of(fn, *args):
    with pytest.raises(YmError) as e:
        fn(*args)
    return e.value.variant


def unit_quaternions(n, rng):
    q = rng.standard_normal((n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def haar_su3(n, rng):
    z = (rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=1, axis2=2)
    q = q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(q)
    q[:, :, 2] /= det[:, None]   # unit determinant
    return q


def identity_text():
    return K.su2_to_canonical_config((2, 2, 2, 2), np.tile([1.0, 0.0, 0.0, 0.0], (64, 1)))


def test_su2_identity_text_is_the_reference_layout():
    t = identity_text()
    lines = t.split("\n")
    assert lines[:3] == ["YM-SU2-CONFIG-V1", "extents=2,2,2,2", "link_count=64"]
    assert lines[3:-1] == ["3ff0000000000000,0000000000000000,0000000000000000,0000000000000000"] * 64
    assert lines[-1] == "" and t.endswith("\n")


def test_su2_round_trip_is_exact_and_matches_the_oracle():
    rng = np.random.default_rng(0x53)
    ext = (2, 3, 2, 4)
    links = unit_quaternions(int(np.prod(ext)) * 4, rng)
    t = K.su2_to_canonical_config(ext, links)
    assert t == CO.to_canonical_config(CO.SU2_CONFIG_FORMAT_ID, ext, CO.su2_rows(links))
    e2, l2 = K.su2_from_canonical_config(t)
    assert e2 == ext and np.array_equal(l2, links)
    assert K.su2_to_canonical_config(e2, l2) == t


def test_su2_parser_fails_closed_like_the_reference():
    t = identity_text()
    bad = "InvalidConfigurationEncoding"
    D = K.su2_from_canonical_config
    assert variant_of(D, t.replace("3ff0000000000000", "3FF0000000000000", 1)) == bad
    assert variant_of(D, t.replace("3ff0000000000000", "4000000000000000", 1)) == "NonUnitSu2"
    assert variant_of(D, f"YM-SU2-CONFIG-V1\nextents=2,2,2,2\nlink_count={2**20 + 1}\n") == "LatticeTooLarge"
    assert variant_of(D, t.replace("3ff0000000000000", "7ff8000000000000", 1)) == "NonFiniteSu2Component"
    assert variant_of(D, t.replace("\n", "\r\n")) == bad           # not the canonical re-encoding
    assert variant_of(D, t[:-1]) == bad                            # final newline missing
    assert variant_of(D, t + "\n") == bad                          # an extra line
    assert variant_of(D, t.replace("extents=2,2,2,2", "extents=+2,2,2,2")) == bad
    assert variant_of(D, t.replace("extents=2,2,2,2", "extents=02,2,2,2")) == bad
    assert variant_of(D, t.replace("extents=2,2,2,2", "extents=2,2,2")) == bad
    assert variant_of(D, t.replace("extents=2,2,2,2", "extents=2,2,2,2,")) == bad
    assert variant_of(D, t.replace("extents=2,2,2,2", "extents=1,2,2,2")) == "InvalidLatticeExtent"
    assert variant_of(D, t.replace("link_count=64", "link_count=63")) == bad
    assert variant_of(D, t.replace("YM-SU2-CONFIG-V1", "YM-SU2-CONFIG-V2")) == bad
    assert variant_of(D, t.replace(",0000000000000000\n", ",000000000000000\n", 1)) == bad
    assert variant_of(D, t.replace(",0000000000000000\n", ",0000000000000000,0\n", 1)) == bad
    assert variant_of(D, "") == bad
    # the same text with a '+' but otherwise parsable still reaches the lattice checks first
    assert variant_of(D, t.replace("extents=2,2,2,2", "extents=+1,2,2,2")) == "InvalidLatticeExtent"
    # encoder refuses non-unit links and lattices over the reference cap
    links = np.tile([1.0, 0.0, 0.0, 0.0], (64, 1))
    links[5] = [1.0, 1e-5, 0.0, 0.0]
    assert variant_of(K.su2_to_canonical_config, (2, 2, 2, 2), links) == "NonUnitSu2"
    big = np.tile([1.0, 0.0, 0.0, 0.0], (2 ** 21, 1))   # 2^21 links > the 2^20 cap
    assert variant_of(K.su2_to_canonical_config, (32, 32, 16, 32), big) == "LatticeTooLarge"


def test_su3_round_trip_and_gates():
    rng = np.random.default_rng(0x33)
    ext = (2, 2, 2, 3)
    links = haar_su3(int(np.prod(ext)) * 4, rng)
    t = K.su3_to_canonical_config(ext, links)
    assert t == CO.to_canonical_config(CO.SU3_CONFIG_FORMAT_ID, ext, CO.su3_rows(links))
    e2, l2 = K.su3_from_canonical_config(t)
    assert e2 == ext and np.array_equal(l2, links)
    bad = links.copy()
    bad[3] *= 1.0 + 1e-9
    assert variant_of(K.su3_to_canonical_config, ext, bad) == "NonUnitaryMatrix"
    bad = links.copy()
    bad[7] *= np.exp(0.1j)   # unitary, det = e^{0.3 i}
    assert variant_of(K.su3_to_canonical_config, ext, bad) == "DeterminantNotOne"
    bad = links.copy()
    bad[0, 1, 2] = np.nan
    assert variant_of(K.su3_to_canonical_config, ext, bad) == "NonFiniteMatrix"
    # decode gates the same way
    text_bad = CO.to_canonical_config(CO.SU3_CONFIG_FORMAT_ID, ext,
                                      CO.su3_rows(np.where(np.arange(len(links))[:, None, None] == 7,
                                                           links * np.exp(0.1j), links)))
    assert variant_of(K.su3_from_canonical_config, text_bad) == "DeterminantNotOne"
    big = np.tile(np.eye(3, dtype=np.complex128), (2 ** 19, 1, 1))   # 2^19 links > the 2^18 cap
    assert variant_of(K.su3_to_canonical_config, (16, 16, 16, 32), big) == "LatticeTooLarge"
    assert variant_of(K.su3_from_canonical_config, t.replace("YM-SU3", "YM-SU2", 1)) == \
        "InvalidConfigurationEncoding"
