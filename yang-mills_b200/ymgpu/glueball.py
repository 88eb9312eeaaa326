"""Glueball measurement path -- mirror of the reference modules
``glueball_operators``, ``glueball_smearing``, ``glueball_blocking``,
``glueball_correlators`` and the correlator/jackknife steps of
``glueball_scalar_production`` / ``glueball_scalar_fit``.

Lattice work (smearing, blocking, operator basis) runs on the device over
every chain of an ``Ensemble`` at once; the correlator, jackknife and
covariance steps are the reference's host FP64 arithmetic in libymgpu.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List

import numpy as np

from ._lib import lib
from .ensemble import Ensemble
from .errors import VARIANTS, YmError, check

EUCLIDEAN_TIME_DIRECTION = 3
SPATIAL_DIRECTIONS = (0, 1, 2)
MINIMUM_SPATIAL_EXTENT = 3
CANONICAL_RHO = 0.10
MAX_RHO = 0.25
MAX_LEVELS = 8
BLOCK_FACTOR = 2
MAX_CONFIGURATIONS = 64
MAX_TIME_EXTENT = 64

_P = C.POINTER(C.c_double)


@dataclass
class ScalarOperatorBasis:
    """glueball_operators.rs:28-34."""
    spatial_plaquette_1x1: float
    spatial_rectangle_2x1: float
    plaquette_loop_count: int
    rectangle_loop_count: int


def scalar_a1pp_operator_basis(ens: Ensemble, chain: int, time_slice: int) -> ScalarOperatorBasis:
    """glueball_operators.rs:143-160 for one chain and time slice."""
    ext = ens.extents[chain]
    if time_slice < 0 or time_slice >= ext[EUCLIDEAN_TIME_DIRECTION]:
        raise YmError(VARIANTS["TimeSliceOutOfRange"], "scalar_a1pp_operator_basis")
    p, r = ens.scalar_operator_basis()[chain]
    vs = ext[0] * ext[1] * ext[2]
    return ScalarOperatorBasis(float(p[time_slice]), float(r[time_slice]), 3 * vs, 6 * vs)


def spatial_stout_smear(ens: Ensemble, rho: float, levels: int,
                        lift_level_cap: bool = False) -> Ensemble:
    """glueball_smearing.rs:257-268: a new handle holding the smeared links."""
    out = ens.like()
    try:
        ens.stout_smear_into(out, rho, levels, lift_level_cap)
    except Exception:
        out.close()
        raise
    return out


def blocked_extents(extents) -> tuple:
    """glueball_blocking.rs:85-94."""
    e = list(extents)
    if e[0] != e[1] or e[1] != e[2]:
        raise YmError(VARIANTS["SpatialExtentsNotCubic"], "blocked_extents")
    if e[0] < BLOCK_FACTOR * MINIMUM_SPATIAL_EXTENT:
        raise YmError(VARIANTS["SpatialExtentTooSmall"], "blocked_extents")
    if e[0] % BLOCK_FACTOR:
        raise YmError(VARIANTS["SpatialExtentNotEven"], "blocked_extents")
    return (e[0] // 2, e[1] // 2, e[2] // 2, e[3])


def spatial_stride2_block(ens: Ensemble) -> Ensemble:
    """glueball_blocking.rs:105-136: a new handle with the coarse lattices."""
    out = ens.like([blocked_extents(e) for e in ens.extents])
    try:
        ens.block_into(out)
    except Exception:
        out.close()
        raise
    return out


# ---------------------------------------------------------------- correlators

def periodic_connected_estimator(samples: np.ndarray):
    """glueball_correlators.rs:111-172: (vacuum mean, raw C(tau), connected C(tau))."""
    s = np.ascontiguousarray(samples, np.float64)
    ncfg, nt = s.shape
    vac = C.c_double()
    raw, con = np.zeros(nt), np.zeros(nt)
    check(lib().ym_periodic_connected_estimator(s.ctypes.data_as(_P), ncfg, nt, C.byref(vac),
                                                raw.ctypes.data_as(_P), con.ctypes.data_as(_P)),
          "periodic_connected_estimator")
    return vac.value, raw, con


def connected_from_samples(samples: np.ndarray, omitted=None) -> np.ndarray:
    """glueball_scalar_production.rs:383-443."""
    s = np.ascontiguousarray(samples, np.float64)
    ncfg, nt = s.shape
    con = np.zeros(nt)
    check(lib().ym_connected_from_samples(s.ctypes.data_as(_P), ncfg, nt,
                                          -1 if omitted is None else int(omitted),
                                          con.ctypes.data_as(_P)), "connected_from_samples")
    return con


def jackknife_replicas(samples: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(samples, np.float64)
    ncfg, nt = s.shape
    out = np.zeros((ncfg, nt))
    check(lib().ym_jackknife_replicas(s.ctypes.data_as(_P), ncfg, nt, out.ctypes.data_as(_P)),
          "jackknife_replicas")
    return out


def jackknife_covariance(replicas: np.ndarray, start: int, end: int) -> np.ndarray:
    """glueball_scalar_fit.rs:276-322 over the window [start, end]."""
    r = np.ascontiguousarray(replicas, np.float64)
    nrep, nt = r.shape
    pts = end - start + 1
    out = np.zeros((pts, pts))
    check(lib().ym_jackknife_covariance(r.ctypes.data_as(_P), nrep, nt, start, end,
                                        out.ctypes.data_as(_P)), "jackknife_covariance")
    return out


@dataclass
class ScalarConnectedCorrelators:
    """glueball_correlators.rs:35-45."""
    configuration_count: int
    time_extent: int
    plaquette_vacuum_mean: float
    rectangle_vacuum_mean: float
    plaquette_raw: np.ndarray
    rectangle_raw: np.ndarray
    plaquette_connected: np.ndarray
    rectangle_connected: np.ndarray


def operator_samples(ens: Ensemble):
    """The configuration x time operator samples of every chain (each chain
    one configuration) -- glueball_scalar_production.rs:338-381."""
    basis = ens.scalar_operator_basis()
    return (np.stack([b[0] for b in basis]), np.stack([b[1] for b in basis]))


def scalar_connected_correlators(ens: Ensemble, lift_configuration_cap: bool = False
                                 ) -> ScalarConnectedCorrelators:
    """glueball_correlators.rs:179-235 with the chains of ``ens`` as the
    configurations (all of one extent)."""
    if ens.n_chains == 0:
        raise YmError(VARIANTS["EmptyConfigurationSet"], "scalar_connected_correlators")
    if ens.n_chains > MAX_CONFIGURATIONS and not lift_configuration_cap:
        raise YmError(VARIANTS["TooManyConfigurations"], "scalar_connected_correlators")
    nt = ens.extents[0][3]
    if nt > MAX_TIME_EXTENT:
        raise YmError(VARIANTS["TimeExtentTooLarge"], "scalar_connected_correlators")
    if any(e != ens.extents[0] for e in ens.extents):
        raise YmError(VARIANTS["LatticeExtentsMismatch"], "scalar_connected_correlators")
    p, r = operator_samples(ens)
    pv, praw, pcon = periodic_connected_estimator(p)
    rv, rraw, rcon = periodic_connected_estimator(r)
    return ScalarConnectedCorrelators(ens.n_chains, nt, pv, rv, praw, rraw, pcon, rcon)
