"""``path_holonomy`` -- mirror of reference/rust/src/path_holonomy.rs on
device-resident lattices.

A path is a list of oriented steps, encoded as integers: ``forward(d)`` =
d + 1 steps from x to x + d, ``backward(d)`` = -(d + 1) steps from x to x - d
and multiplies by the dagger of the link there (``OrientedStep``,
path_holonomy.rs:19-45).  Holonomies are products in traversal order from the
left, each one the reference's checked SU(3) product, evaluated by the engine
(``include/ymgpu.h``).  ``lattice`` is a ``Su3Lattice4`` or ``Lattice4``.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from ._lib import lib
from .errors import check

MAX_PATH_STEPS = 1 << 20          # path_holonomy.rs:17


def forward(direction: int) -> int:
    return direction + 1


def backward(direction: int) -> int:
    return -(direction + 1)


def reversed_step(step: int) -> int:
    """OrientedStep::reversed (path_holonomy.rs:38-44)."""
    return -step


def rectangular_path(mu: int, nu: int, r: int, t: int) -> List[int]:
    """path_holonomy.rs:219-260: R forward along mu, T forward along nu, R
    back, T back (validated by the engine in the reference's order)."""
    cap = max(0, 2 * (int(r) + int(t)))
    buf = np.zeros(max(cap, 1), np.int32)
    n = C.c_int64()
    check(lib().ym_rectangular_path(int(mu), int(nu), int(r), int(t),
                                    buf.ctypes.data_as(C.POINTER(C.c_int32)), buf.size, C.byref(n)),
          "rectangular_path")
    return [int(v) for v in buf[:n.value]]


def reverse_path(steps: Sequence[int]) -> List[int]:
    """path_holonomy.rs:183-196: the steps in reverse order, each reversed."""
    _validate(steps)
    return [reversed_step(s) for s in reversed(list(steps))]


def concatenate_paths(first: Sequence[int], second: Sequence[int]) -> List[int]:
    """path_holonomy.rs:198-217."""
    _validate(first)
    _validate(second)
    if len(first) + len(second) > MAX_PATH_STEPS:
        from .errors import VARIANTS, YmError
        raise YmError(VARIANTS["PathTooLong"], "concatenate_paths")
    return list(first) + list(second)


def _validate(steps: Sequence[int]) -> None:
    from .errors import VARIANTS, YmError
    if len(steps) == 0:
        raise YmError(VARIANTS["EmptyPath"], "path")
    if len(steps) > MAX_PATH_STEPS:
        raise YmError(VARIANTS["PathTooLong"], "path")
    if any(s == 0 or abs(s) > 4 for s in steps):
        raise YmError(VARIANTS["DirectionOutOfRange"], "path")


def _target(lattice):
    return lattice.ensemble, 0


def path_holonomy(lattice, start, steps):
    """(holonomy, end) along steps from start (path_holonomy.rs:132-161)."""
    ens, chain = _target(lattice)
    return ens.path_holonomy(chain, start, steps)


def closed_path_holonomy(lattice, start, steps):
    """path_holonomy.rs:163-170: PathNotClosed unless the path returns to start."""
    hol, end = path_holonomy(lattice, start, steps)
    if tuple(int(v) for v in start) != end:
        from .errors import VARIANTS, YmError
        raise YmError(VARIANTS["PathNotClosed"], "closed_path_holonomy")
    return hol


def wilson_loop(lattice, start, steps) -> complex:
    """(1/3) Tr of the closed holonomy (path_holonomy.rs:172-181)."""
    ens, chain = _target(lattice)
    return ens.wilson_loop(chain, start, steps)


def wilson_loop_sites(lattice, steps) -> np.ndarray:
    """wilson_loop of the same closed path from every site (lexicographic)."""
    ens, chain = _target(lattice)
    return ens.wilson_loop_sites(chain, steps)
