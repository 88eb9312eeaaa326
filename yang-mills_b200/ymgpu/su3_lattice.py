"""Device-resident ``Su3Lattice4`` -- mirror of the reference type
(reference/rust/src/su3_lattice.rs:20-313).

The links live on the GPU in the engine's structure-of-arrays layout; every
method evaluates on the device and moves only its result (one link for
link/set_link, one matrix for plaquette, one number for the action).
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from .ensemble import Ensemble

DIM = 4


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
        """su3_lattice.rs:153-155: one link (3, 3) complex128, moved alone."""
        return self.ensemble.get_link(0, x, mu)

    def set_link(self, x, mu: int, value: np.ndarray) -> None:
        """su3_lattice.rs:157-166: one link, moved alone."""
        self.ensemble.set_link(0, x, mu, value)

    def plaquette(self, x, mu: int, nu: int) -> np.ndarray:
        """su3_lattice.rs:168-181 (checked products)."""
        return self.ensemble.plaquette_at(0, x, mu, nu)

    def polyakov_holonomy(self, start, direction: int) -> np.ndarray:
        """su3_lattice.rs:185-200: the ordered product wrapping one extent."""
        n = self.extents()[direction]
        hol, _ = self.ensemble.path_holonomy(0, start, [direction + 1] * n)
        return hol

    def polyakov_loop(self, start, direction: int) -> complex:
        """su3_lattice.rs:202-212: (1/3) Tr of the periodic holonomy."""
        return self.ensemble.polyakov_loop(0, start, direction)

    def wilson_action(self, beta: float) -> float:
        """su3_lattice.rs:214-242 (the reference's sequential sum)."""
        return float(self.ensemble.wilson_action(beta)[0])

    def gauge_transform(self, omega) -> "Su3Lattice4":
        """su3_lattice.rs:244-283: a new lattice with g(x) U_mu(x) g(x+mu)^dag;
        omega is a callable x -> (3, 3) matrix or a (V, 3, 3) array of
        per-site gauges in lexicographic order."""
        ext = self.extents()
        if callable(omega):
            g = np.empty((self.site_count(), 3, 3), np.complex128)
            k = 0
            for x0 in range(ext[0]):
                for x1 in range(ext[1]):
                    for x2 in range(ext[2]):
                        for x3 in range(ext[3]):
                            g[k] = omega((x0, x1, x2, x3))
                            k += 1
        else:
            g = np.asarray(omega, dtype=np.complex128)
        out = Su3Lattice4(self.ensemble.like())
        self.ensemble.gauge_transform(0, g, out.ensemble, 0)
        return out

    def max_link_unitarity_residual(self) -> float:
        return float(self.ensemble.max_residuals()[0][0])

    def max_link_determinant_residual(self) -> float:
        return float(self.ensemble.max_residuals()[1][0])

    def close(self) -> None:
        self.ensemble.close()
