"""Device-resident ``Lattice4`` -- mirror of the reference's SU(2) lattice
(reference/rust/src/lib.rs:235-546).

Links are unit quaternions (a0, a1, a2, a3), U = a0 I - i a.sigma, held on
the GPU; every method evaluates on the device with the reference's products
(each re-normalised as Su2::mul does) and moves only its result.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from .ensemble import SU2, Ensemble
from .path_holonomy import rectangular_path

DIM = 4


class Lattice4:
    """One SU(2) lattice held on the device (a one-chain ``Ensemble``)."""

    def __init__(self, ensemble: Ensemble):
        if ensemble.group != SU2:
            raise ValueError("Lattice4 holds an SU(2) ensemble")
        self.ensemble = ensemble

    @classmethod
    def new_identity(cls, extents: Sequence[int], lift_reference_caps: bool = False,
                     device: int = 0) -> "Lattice4":
        """lib.rs:242-262 (every link the identity)."""
        return cls(Ensemble([list(extents)], 0.0, 0, group=SU2,
                            lift_reference_caps=lift_reference_caps, device=device))

    @classmethod
    def from_links(cls, extents, links: np.ndarray, **kw) -> "Lattice4":
        lat = cls.new_identity(extents, **kw)
        lat.ensemble.upload(0, links)
        return lat

    def extents(self):
        return self.ensemble.extents[0]

    def site_count(self) -> int:
        return int(np.prod(self.extents()))

    def links(self) -> np.ndarray:
        """All links, (links, 4) float64 in the reference layout."""
        return self.ensemble.download(0)

    def link(self, x, mu: int) -> np.ndarray:
        return self.ensemble.get_link(0, x, mu)

    def set_link(self, x, mu: int, value) -> None:
        self.ensemble.set_link(0, x, mu, value)

    def plaquette(self, x, mu: int, nu: int) -> np.ndarray:
        """lib.rs:348-361."""
        return self.ensemble.plaquette_at(0, x, mu, nu)

    def wilson_action(self, beta: float) -> float:
        """lib.rs:363-382."""
        return float(self.ensemble.wilson_action(beta)[0])

    def staple(self, x, mu: int):
        """lib.rs:507-546: (components, terms)."""
        return self.ensemble.su2_staple(0, x, mu)

    def path_holonomy(self, start, steps):
        return self.ensemble.path_holonomy(0, start, steps)

    def wilson_loop(self, start, steps) -> float:
        """lib.rs:430-436: half real trace of the closed holonomy."""
        return self.ensemble.wilson_loop(0, start, steps).real

    @staticmethod
    def rectangular_path(mu: int, nu: int, r: int, t: int):
        return rectangular_path(mu, nu, r, t)

    def rectangular_wilson_loop(self, start, mu: int, nu: int, r: int, t: int) -> float:
        """lib.rs:471-481."""
        return self.wilson_loop(start, rectangular_path(mu, nu, r, t))

    def polyakov_loop(self, start, direction: int) -> float:
        """lib.rs:483-505."""
        return self.ensemble.polyakov_loop(0, start, direction).real

    def max_link_unit_residual(self) -> float:
        return float(self.ensemble.max_unit_residual()[0])

    def close(self) -> None:
        self.ensemble.close()
