"""Stream and statistics helpers shared by the SU(2) and SU(3) ensembles --
mirror of the reference module ``su2_ensemble`` (su2_ensemble.rs:24-55,
375-463) and of ``sampling_efficiency::evaluate`` (sampling_efficiency.rs:57-135).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import ChainDiagnostics as _CDiag
from ._lib import EfficiencyReport as _CEff
from ._lib import lib
from .errors import check

RNG_ID = "SPLITMIX64-V1"


def derive_chain_seed(master_seed: int, chain_id: int) -> int:
    return lib().ym_derive_chain_seed(master_seed, chain_id)


def splitmix64_at(seed: int, n: int) -> int:
    """Output n (0-based) of the reference SplitMix64 stream seeded with ``seed``."""
    return lib().ym_splitmix64_at(seed, n)


@dataclass
class SweepStream:
    """Counter-based replacement of the reference's ``&mut SplitMix64``: the
    chain seed plus the index of the next sweep.  Sweep n keys link (x, mu)
    with S(S(seed, n), 4*site+mu), S(k, i) = output i of SplitMix64::new(k)."""
    seed: int
    sweep: int = 0


@dataclass
class ChainDiagnostics:
    mean: float
    variance: float
    autocorrelation: np.ndarray
    positive_window_lag: int
    integrated_autocorrelation_time: float
    effective_sample_size: float
    standard_error: float


def diagnostics(values, max_lag: int):
    v = np.ascontiguousarray(values, np.float64)
    ac = np.zeros(max_lag + 1, np.float64)
    out = _CDiag()
    check(lib().ym_diagnostics(v.ctypes.data_as(C.POINTER(C.c_double)), len(v), max_lag,
                               C.byref(out), ac.ctypes.data_as(C.POINTER(C.c_double))),
          "diagnostics")
    d = ChainDiagnostics(out.mean, out.variance, ac, out.positive_window_lag,
                         out.integrated_autocorrelation_time, out.effective_sample_size,
                         out.standard_error)
    return d, ac


@dataclass
class EfficiencyReport:
    diagnostics: ChainDiagnostics
    reweighting_efficiency: float
    weight_only_ess: float
    combined_ess_proxy: float
    total_cost: float
    sampling_cost_per_effective_sample_proxy: float
    total_cost_per_effective_sample_proxy: float


def sampling_efficiency(values, log_weights, max_lag, setup, thermalization, sampling):
    """``sampling_efficiency::evaluate`` with SamplingCost(setup, thermalization, sampling)."""
    v = np.ascontiguousarray(values, np.float64)
    w = None if log_weights is None else np.ascontiguousarray(log_weights, np.float64)
    ac = np.zeros(max_lag + 1, np.float64)
    out = _CEff()
    P = C.POINTER(C.c_double)
    check(lib().ym_sampling_efficiency(v.ctypes.data_as(P), len(v),
                                       None if w is None else w.ctypes.data_as(P), max_lag,
                                       setup, thermalization, sampling, C.byref(out),
                                       ac.ctypes.data_as(P)), "sampling_efficiency")
    d = out.diagnostics
    diag = ChainDiagnostics(d.mean, d.variance, ac, d.positive_window_lag,
                            d.integrated_autocorrelation_time, d.effective_sample_size,
                            d.standard_error)
    return EfficiencyReport(diag, out.reweighting_efficiency, out.weight_only_ess,
                            out.combined_ess_proxy, out.total_cost,
                            out.sampling_cost_per_effective_sample_proxy,
                            out.total_cost_per_effective_sample_proxy)


# ---------------------------------------------------------------- SU(2) chains

SAMPLER_ID = "YM-SU2-ENSEMBLE-V1"
MAX_REFERENCE_BETA = 8.0
MAX_REFERENCE_SWEEPS = 1 << 20
MAX_REFERENCE_MEASUREMENTS = 1 << 20
MAX_OVERRELAXATION_SWEEPS = 16
MAX_REFERENCE_LINKS = 1 << 20


def _err(name: str, where: str):
    from .errors import VARIANTS, YmError
    return YmError(VARIANTS[name], where)


@dataclass
class EnsembleConfig:
    """su2_ensemble.rs:57-107."""
    extents: tuple
    beta: float
    master_seed: int
    chain_id: int
    thermalization_sweeps: int
    measurements: int
    sweeps_between_measurements: int
    overrelaxation_sweeps_per_heatbath: int
    max_heatbath_attempts_per_link: int
    autocorrelation_max_lag: int

    def validate(self) -> "EnsembleConfig":
        if not np.isfinite(self.beta) or self.beta < 0.0 or self.beta > MAX_REFERENCE_BETA:
            raise _err("BetaOutsideReferenceRange", "validate")
        if self.measurements > MAX_REFERENCE_MEASUREMENTS:
            raise _err("ScheduleOutsideReferenceRange", "validate")
        total = self.thermalization_sweeps + self.measurements * self.sweeps_between_measurements
        if total > MAX_REFERENCE_SWEEPS:
            raise _err("ScheduleOutsideReferenceRange", "validate")
        if self.measurements < 2:
            raise _err("TooFewMeasurements", "validate")
        if self.sweeps_between_measurements == 0:
            raise _err("ZeroMeasurementStride", "validate")
        if self.overrelaxation_sweeps_per_heatbath > MAX_OVERRELAXATION_SWEEPS:
            raise _err("TooManyOverrelaxationSweeps", "validate")
        if self.max_heatbath_attempts_per_link == 0:
            raise _err("ZeroHeatbathAttemptLimit", "validate")
        if self.autocorrelation_max_lag >= self.measurements:
            raise _err("AutocorrelationLagOutOfRange", "validate")
        return self


@dataclass
class ChainReport:
    """su2_ensemble.rs:172-186."""
    config: EnsembleConfig
    derived_seed: int
    total_heatbath_sweeps: int
    total_overrelaxation_sweeps: int
    heatbath_proposals: int
    heatbath_updates: int
    mean_heatbath_acceptance: float
    measurements: np.ndarray
    diagnostics: ChainDiagnostics
    final_link_unit_residual: float
    sampler_id: str = SAMPLER_ID
    rng_id: str = RNG_ID


def run_chains(configs, sampler: str = "reference", device: int = 0):
    """``run_chain`` (su2_ensemble.rs:488-552) for many chains of one schedule
    in the same device launches; cold start, heat-bath + overrelaxation."""
    from .ensemble import SU2, Ensemble
    for c in configs:
        c.validate()
    sched = {(c.thermalization_sweeps, c.measurements, c.sweeps_between_measurements,
              c.overrelaxation_sweeps_per_heatbath, c.max_heatbath_attempts_per_link)
             for c in configs}
    if len(sched) != 1:
        raise ValueError("run_chains needs one common schedule")
    therm, nmeas, stride, n_or, attempts = sched.pop()
    seeds = [derive_chain_seed(c.master_seed, c.chain_id) for c in configs]
    ens = Ensemble([list(c.extents) for c in configs], [c.beta for c in configs], seeds,
                   group=SU2, device=device)
    try:
        ens.markov_sweeps(therm, n_or, attempts, sampler)
        # measurement m after `stride` more sweeps, all on the device
        # (ym_su2_measured_sweeps: the values of the separate calls)
        meas = ens.su2_measured_sweeps(nmeas, stride, n_or, attempts, sampler).T.copy()
        prop, upd = ens.heatbath_accounting()
        res = ens.max_unit_residual()
    finally:
        ens.close()
    total = therm + nmeas * stride
    out = []
    for i, c in enumerate(configs):
        diag, _ = diagnostics(meas[i], c.autocorrelation_max_lag)
        out.append(ChainReport(c, seeds[i], total, total * n_or, int(prop[i]), int(upd[i]),
                               float(upd[i]) / float(prop[i]), meas[i], diag, float(res[i])))
    return out


def run_chain(config: EnsembleConfig, **kw) -> ChainReport:
    return run_chains([config], **kw)[0]
