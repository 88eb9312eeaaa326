"""Batched campaign drivers built from the engine's entry points.

``batched_su3_chains``: many independent SU(3) Metropolis chains in one
handle (every sub-sweep launch covers all of them), the run_chain cadence
(su3_ensemble.rs:408-480) replayed from a captured graph, per-chain
diagnostics through the reference estimator.

``scalar_glueball_pipeline``: uneven chain groups in one handle, then per
measurement spatial stout smearing at several level counts, stride-2
blocking where the reference admits it (fine extent >= 6 and even), the A1++
operator basis per time slice, connected correlators, delete-one jackknife
replicas and the jackknife covariance -- the production cadence of
glueball_scalar_production.rs:257-472 with every lattice step on the device.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import glueball as G
from .ensemble import F64, Ensemble
from .su2_ensemble import diagnostics
from .su3_ensemble import derive_su3_chain_seed


@dataclass
class BatchedChainsResult:
    series: np.ndarray                 # [chain, measurement]
    effective_sample_size: np.ndarray  # per chain
    integrated_autocorrelation_time: np.ndarray
    pooled_mean: float
    pooled_error: float
    acceptance: float
    link_updates: int
    seconds: float

    @property
    def link_updates_per_s(self) -> float:
        return self.link_updates / self.seconds

    @property
    def ess_per_s(self) -> float:
        return float(np.sum(self.effective_sample_size)) / self.seconds


def batched_su3_chains(n_chains: int = 64, extents=(4, 4, 4, 4), beta: float = 6.0,
                       master_seed: int = 0x2C02198105010002, thermalization: int = 0,
                       measurements: int = 1000, sweeps_per_measurement: int = 1,
                       proposal_angle: float = 0.3, generator_mode: str = "uniform",
                       max_lag: int = 50, precision: int = F64, device: int = 0
                       ) -> BatchedChainsResult:
    seeds = [derive_su3_chain_seed(master_seed, i) for i in range(n_chains)]
    with Ensemble([list(extents)] * n_chains, beta, seeds, precision=precision,
                  lift_reference_caps=True, device=device) as ens:
        if thermalization:
            ens.metropolis_sweeps(proposal_angle, thermalization, generator_mode)
        ens.synchronize()
        p0, a0 = ens.accounting()
        t0 = time.perf_counter()
        series = ens.measured_sweeps(proposal_angle, measurements, sweeps_per_measurement,
                                     generator_mode).T.copy()
        secs = time.perf_counter() - t0
        p1, a1 = ens.accounting()
    lag = max(1, min(max_lag, measurements - 1))
    diags = [diagnostics(series[c], lag)[0] for c in range(n_chains)]
    means = series.mean(1)
    return BatchedChainsResult(
        series=series,
        effective_sample_size=np.array([d.effective_sample_size for d in diags]),
        integrated_autocorrelation_time=np.array([d.integrated_autocorrelation_time for d in diags]),
        pooled_mean=float(means.mean()),
        pooled_error=float(means.std(ddof=1) / np.sqrt(n_chains)) if n_chains > 1 else float("nan"),
        acceptance=float((a1 - a0).sum()) / float((p1 - p0).sum()),
        link_updates=int(n_chains * int(np.prod(extents)) * 4 * measurements * sweeps_per_measurement),
        seconds=secs)


@dataclass
class SurfaceResult:
    """One (group, stout levels, blocked) correlator surface."""
    extents: Tuple[int, ...]
    stout_levels: int
    blocked: bool
    plaquette_samples: np.ndarray      # [configuration, t]
    rectangle_samples: np.ndarray
    plaquette_connected: np.ndarray    # C(tau)
    rectangle_connected: np.ndarray
    plaquette_jackknife: np.ndarray    # [replica, tau]
    plaquette_covariance: np.ndarray   # over tau in [1, min(4, T/2)]


@dataclass
class GlueballPipelineResult:
    surfaces: List[SurfaceResult] = field(default_factory=list)
    sweep_seconds: float = 0.0
    measure_seconds: float = 0.0
    link_updates: int = 0


def _blockable(e) -> bool:
    return e[0] == e[1] == e[2] and e[0] >= 6 and e[0] % 2 == 0


def scalar_glueball_pipeline(groups: Sequence[Tuple[int, Sequence[int]]] = ((128, (4, 4, 4, 10)),
                                                                           (64, (6, 6, 6, 12)),
                                                                           (32, (8, 8, 8, 16))),
                             beta: float = 5.7, master_seed: int = 0x3F00202609150001,
                             thermalization: int = 64, measurements: int = 4,
                             sweeps_between_measurements: int = 4, proposal_angle: float = 0.35,
                             stout_levels: Sequence[int] = (0, 5, 10), rho: float = 0.1,
                             device: int = 0) -> GlueballPipelineResult:
    """Every chain of every group evolves in the same launches; the samples of
    each group (chains x measurements configurations) feed its correlators."""
    extents, group_of = [], []
    for gi, (count, ext) in enumerate(groups):
        extents += [list(ext)] * count
        group_of += [gi] * count
    seeds = [derive_su3_chain_seed(master_seed, i) for i in range(len(extents))]
    res = GlueballPipelineResult()
    samples: Dict[Tuple[int, int, bool], List[Tuple[np.ndarray, np.ndarray]]] = {}
    with Ensemble(extents, beta, seeds, lift_reference_caps=True, device=device) as ens:
        per_group = [[i for i, g in enumerate(group_of) if g == gi] for gi in range(len(groups))]
        # Scratch handles made once and refilled every measurement: the
        # smeared copy of all chains, and per blockable group its chains and
        # their blocked lattices.
        sm = ens.like()
        subs, coarse = {}, {}
        for gi, chains in enumerate(per_group):
            if _blockable(groups[gi][1]):
                subs[gi] = sm.subset(chains)
                coarse[gi] = subs[gi].like([G.blocked_extents(e) for e in subs[gi].extents])
        try:
            t0 = time.perf_counter()
            ens.metropolis_sweeps(proposal_angle, thermalization)
            ens.synchronize()
            res.sweep_seconds += time.perf_counter() - t0
            for _ in range(measurements):
                t0 = time.perf_counter()
                ens.metropolis_sweeps(proposal_angle, sweeps_between_measurements)
                ens.synchronize()
                t1 = time.perf_counter()
                res.sweep_seconds += t1 - t0
                for levels in stout_levels:
                    ens.stout_smear_into(sm, rho, levels, lift_level_cap=True)
                    basis = sm.scalar_operator_basis()
                    for gi, chains in enumerate(per_group):
                        samples.setdefault((gi, levels, False), []).extend(basis[c] for c in chains)
                        if gi in subs:
                            sm.copy_subset_to(chains, subs[gi])
                            subs[gi].block_into(coarse[gi])
                            samples.setdefault((gi, levels, True), []).extend(
                                coarse[gi].scalar_operator_basis())
                res.measure_seconds += time.perf_counter() - t1
        finally:
            for h in list(coarse.values()) + list(subs.values()) + [sm]:
                h.close()
        res.link_updates = int(sum(np.prod(e) * 4 for e in extents)) * (
            thermalization + measurements * sweeps_between_measurements)
    for (gi, levels, blocked), rows in sorted(samples.items()):
        p = np.stack([r[0] for r in rows])
        r = np.stack([r[1] for r in rows])
        nt = p.shape[1]
        reps = G.jackknife_replicas(p)
        end = min(4, nt // 2)
        cov = G.jackknife_covariance(reps, 1, end) if len(reps) > end else np.zeros((0, 0))
        res.surfaces.append(SurfaceResult(
            tuple(groups[gi][1]) if not blocked else G.blocked_extents(groups[gi][1]),
            levels, blocked, p, r, G.connected_from_samples(p), G.connected_from_samples(r),
            reps, cov))
    return res
