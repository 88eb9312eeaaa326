"""SU(3) Metropolis ensembles on the device -- mirror of the reference module
``su3_ensemble`` (reference/rust/src/su3_ensemble.rs).

Same names, argument meanings and fail-closed checks as the reference:
``Su3EnsembleConfig.validate`` (:58-97), ``run_chain`` (:408-480),
``metropolis_sweep`` (:342-391), ``average_plaquette`` (:228-259),
``derive_su3_chain_seed`` (:189-192), ``proposal_angle_from_u64`` (:199-213).
The sweep runs on the GPU over an even/odd checkerboard; the reference's
``&mut SplitMix64`` becomes a ``SweepStream`` (seed plus sweep counter) that
keys one counter-based SplitMix64 stream per link visit.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from ._lib import lib
from .errors import YmError, VARIANTS, check
from .ensemble import Ensemble
from .su2_ensemble import ChainDiagnostics, SweepStream, diagnostics
from .su3_lattice import Su3Lattice4

SAMPLER_ID = "YM-SU3-ENSEMBLE-V1"
PROPOSAL_ID = "YM-SU3-GENERATOR-METROPOLIS-V1"
RNG_ID = "SPLITMIX64-V1"
STREAM_ID = "YM-SU3-STREAM-V1"
STREAM_DOMAIN = 0x535533454E535631
MAX_REFERENCE_BETA = 12.0
MAX_REFERENCE_SWEEPS = 512
MAX_REFERENCE_MEASUREMENTS = 512
MIN_PROPOSAL_ANGLE = 1.0e-8
MAX_PROPOSAL_ANGLE = 1.0
PLAQUETTE_TOLERANCE = 1.0e-12
LINK_RESIDUAL_LIMIT = 5.0e-12
MAX_SU3_REFERENCE_LINKS = 1 << 18


def _err(name: str, where: str) -> YmError:
    return YmError(VARIANTS[name], where)


def derive_su3_chain_seed(master_seed: int, chain_id: int) -> int:
    return lib().ym_derive_su3_chain_seed(master_seed, chain_id)


def proposal_angle_from_u64(raw: int, proposal_angle: float) -> float:
    out = C.c_double()
    check(lib().ym_proposal_angle_from_u64(raw, proposal_angle, C.byref(out)),
          "proposal_angle_from_u64")
    return out.value


def _validate_angle(a: float) -> None:
    if not np.isfinite(a) or a < MIN_PROPOSAL_ANGLE or a > MAX_PROPOSAL_ANGLE:
        raise _err("ProposalAngleOutsideReferenceRange", "proposal_angle")


@dataclass
class Su3EnsembleConfig:
    extents: Sequence[int]
    beta: float
    master_seed: int
    chain_id: int
    thermalization_sweeps: int
    measurements: int
    sweeps_between_measurements: int
    proposal_angle: float
    autocorrelation_max_lag: int

    def validate(self, lift_reference_caps: bool = False) -> "Su3EnsembleConfig":
        """su3_ensemble.rs:58-97; ``lift_reference_caps`` admits more sweeps,
        measurements and links than the reference's bounded surface."""
        if not np.isfinite(self.beta) or self.beta < 0.0 or self.beta > MAX_REFERENCE_BETA:
            raise _err("BetaOutsideReferenceRange", "validate")
        _validate_angle(self.proposal_angle)
        max_meas = 1 << 40 if lift_reference_caps else MAX_REFERENCE_MEASUREMENTS
        if self.measurements < 2 or self.measurements > max_meas:
            raise _err("MeasurementCountOutsideReferenceRange", "validate")
        if self.sweeps_between_measurements == 0:
            raise _err("ZeroMeasurementStride", "validate")
        if self.autocorrelation_max_lag >= self.measurements:
            raise _err("AutocorrelationLagOutOfRange", "validate")
        total = self.thermalization_sweeps + self.measurements * self.sweeps_between_measurements
        if not lift_reference_caps and total > MAX_REFERENCE_SWEEPS:
            raise _err("ScheduleOutsideReferenceRange", "validate")
        links = int(np.prod(self.extents)) * 4
        if any(n < 2 for n in self.extents) or (not lift_reference_caps and
                                                links > MAX_SU3_REFERENCE_LINKS):
            raise _err("LatticeOutsideReferenceRange", "validate")
        return self


@dataclass
class MetropolisAccounting:
    proposals: int = 0
    accepts: int = 0


@dataclass
class Su3ChainReport:
    config: Su3EnsembleConfig
    derived_seed: int
    total_sweeps: int
    metropolis_proposals: int
    metropolis_accepts: int
    mean_metropolis_acceptance: float
    measurements: np.ndarray
    diagnostics: ChainDiagnostics
    final_link_unitarity_residual: float
    final_link_determinant_residual: float
    sampler_id: str = SAMPLER_ID
    proposal_id: str = PROPOSAL_ID
    rng_id: str = RNG_ID
    stream_id: str = STREAM_ID


def metropolis_sweep(lattice: Su3Lattice4, beta: float, proposal_angle: float,
                     rng: SweepStream, generator_mode="ordered") -> MetropolisAccounting:
    """One checkerboard Metropolis sweep of ``lattice`` on the device."""
    ens = lattice.ensemble
    ens.set_chain(0, beta, rng.seed)
    ens.sweep_index = rng.sweep
    p0, a0 = ens.accounting()
    ens.metropolis_sweeps(proposal_angle, 1, generator_mode)
    p1, a1 = ens.accounting()
    rng.sweep += 1
    return MetropolisAccounting(int(p1[0] - p0[0]), int(a1[0] - a0[0]))


def local_link_action(lattice: Su3Lattice4, x, mu: int, beta: float) -> float:
    """su3_ensemble.rs:311-317."""
    return lattice.ensemble.local_link_action(0, x, mu, beta)


def local_action_difference(lattice: Su3Lattice4, x, mu: int, candidate, beta: float) -> float:
    """su3_ensemble.rs:319-334: S(candidate) - S(current) over the twelve
    plaquettes holding link (x, mu)."""
    return lattice.ensemble.local_action_difference(0, x, mu, candidate, beta)


def average_plaquette(lattice: Su3Lattice4) -> float:
    return float(lattice.ensemble.average_plaquette()[0])


def run_chains(configs: List[Su3EnsembleConfig], lift_reference_caps: bool = False,
               generator_mode="ordered", device: int = 0) -> List[Su3ChainReport]:
    """``run_chain`` for many chains at once: every chain of one schedule runs
    in the same device launches (extents, beta and seeds may differ)."""
    for c in configs:
        c.validate(lift_reference_caps)
    sched = {(c.thermalization_sweeps, c.measurements, c.sweeps_between_measurements,
              c.proposal_angle) for c in configs}
    if len(sched) != 1:
        raise ValueError("run_chains needs one common schedule and proposal angle")
    therm, nmeas, stride, angle = sched.pop()
    seeds = [derive_su3_chain_seed(c.master_seed, c.chain_id) for c in configs]
    ens = Ensemble([list(c.extents) for c in configs], [c.beta for c in configs], seeds,
                   lift_reference_caps=lift_reference_caps, device=device)
    try:
        ens.metropolis_sweeps(angle, therm, generator_mode)
        # measurement m after `stride` more sweeps, all on the device
        # (ym_su3_measured_sweeps: the values of the separate calls)
        meas = ens.measured_sweeps(angle, nmeas, stride, generator_mode).T.copy()
        if np.any(meas < -0.5 - PLAQUETTE_TOLERANCE) or np.any(meas > 1.0 + PLAQUETTE_TOLERANCE):
            raise _err("NonFiniteStatistic", "run_chain")
        prop, acc = ens.accounting()
        ures, dres = ens.max_residuals()
    finally:
        ens.close()
    reports = []
    for i, c in enumerate(configs):
        diag, _ = diagnostics(meas[i], c.autocorrelation_max_lag)
        if ures[i] > LINK_RESIDUAL_LIMIT or dres[i] > LINK_RESIDUAL_LIMIT:
            raise _err("NonFiniteStatistic", "run_chain residual gate")
        reports.append(Su3ChainReport(
            config=c, derived_seed=seeds[i], total_sweeps=therm + nmeas * stride,
            metropolis_proposals=int(prop[i]), metropolis_accepts=int(acc[i]),
            mean_metropolis_acceptance=float(acc[i]) / float(prop[i]),
            measurements=meas[i], diagnostics=diag,
            final_link_unitarity_residual=float(ures[i]),
            final_link_determinant_residual=float(dres[i])))
    return reports


def run_chain(config: Su3EnsembleConfig, **kw) -> Su3ChainReport:
    return run_chains([config], **kw)[0]
