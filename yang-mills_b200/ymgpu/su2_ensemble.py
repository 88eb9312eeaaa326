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
