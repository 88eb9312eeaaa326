"""Device-resident ``Su3Lattice4`` -- mirror of the reference type
(reference/rust/src/su3_lattice.rs:20-313).

The links live on the GPU in the engine's structure-of-arrays layout; the
accessors below move them in the reference's own order when a caller asks.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from .ensemble import Ensemble

DIM = 4


def _site_index(extents, x) -> int:
    return ((x[0] * extents[1] + x[1]) * extents[2] + x[2]) * extents[3] + x[3]


class Su3Lattice4:
    """One SU(3) lattice held on the device (a one-chain ``Ensemble``)."""

    def __init__(self, ensemble: Ensemble):
        self.ensemble = ensemble

    @classmethod
    def new_identity(cls, extents: Sequence[int], lift_reference_caps: bool = False,
                     device: int = 0) -> "Su3Lattice4":
        """su3_lattice.rs:85-106 (cold start; caps enforced unless lifted)."""
        return cls(Ensemble([list(extents)], 0.0, 0, lift_reference_caps=lift_reference_caps,
                            device=device))

    @classmethod
    def from_links(cls, extents, links: np.ndarray, **kw) -> "Su3Lattice4":
        lat = cls.new_identity(extents, **kw)
        lat.ensemble.upload(0, links)
        return lat

    def extents(self):
        return self.ensemble.extents[0]

    def site_count(self) -> int:
        return int(np.prod(self.extents()))

    def link_count(self) -> int:
        return self.site_count() * DIM

    def links(self) -> np.ndarray:
        """All links in the reference layout (link = site*4 + mu)."""
        return self.ensemble.download(0)

    def link(self, x, mu: int) -> np.ndarray:
        return self.links()[_site_index(self.extents(), x) * DIM + mu]

    def set_link(self, x, mu: int, value: np.ndarray) -> None:
        a = self.links()
        a[_site_index(self.extents(), x) * DIM + mu] = value
        self.ensemble.upload(0, a)

    def max_link_unitarity_residual(self) -> float:
        return float(self.ensemble.max_residuals()[0][0])

    def max_link_determinant_residual(self) -> float:
        return float(self.ensemble.max_residuals()[1][0])

    def close(self) -> None:
        self.ensemble.close()
