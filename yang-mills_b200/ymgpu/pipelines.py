"""Batched campaign drivers built from the engine's entry points.

``batched_su3_chains``: many independent SU(3) Metropolis chains in one
handle (every sub-sweep launch covers all of them), the run_chain cadence
(su3_ensemble.rs:408-480) replayed from a captured graph, per-chain
diagnostics through the reference estimator.

``su3_measured_run`` / ``fp32_vs_fp64_run``: the loop-measurement cadence
of large SU(3) lattices -- sweeps with the plaquette after every one, Wilson
loops R x T <= 4 x 4 and Polyakov loops every block of sweeps, each block one
captured graph -- in two-row binary32 (binary64 reunitarisation every sweep)
or binary64 storage, and the binary32 run's error against a binary64 run of
the same length from the same field, seeds and sweep indices.

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
from .ensemble import F32_TWO_ROW, F64, Ensemble
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
class MeasuredRunResult:
    extents: List[Tuple[int, ...]]
    precision: int
    sweeps_per_block: int
    plaquette: np.ndarray              # [sweep, chain]
    wilson: np.ndarray                 # [block, chain, plane, R-1, T-1]
    polyakov: np.ndarray               # [block, chain] complex
    seconds: float                     # the measured run (sweeps + loop measurements)
    sweep_seconds: float               # the same number of sweeps with a plaquette each, no loops
    link_updates: int

    @property
    def link_updates_per_s(self) -> float:
        return self.link_updates / self.seconds

    @property
    def loop_measurement_seconds(self) -> float:
        return max(0.0, self.seconds - self.sweep_seconds)


def su3_measured_run(ens: Ensemble, n_blocks: int, sweeps_per_block: int = 10,
                     proposal_angle: float = 0.3, generator_mode: str = "ordered",
                     rmax: int = 4, tmax: int = 4, polyakov_direction: int = 3,
                     view: Ensemble = None, time_sweeps_alone: bool = True) -> MeasuredRunResult:
    """The loop-measurement cadence on an existing handle (its current field,
    seeds and sweep index).  A two-row handle measures its loops through a
    binary64 ``view`` (made here when not given).  With time_sweeps_alone the
    same sweeps are timed once more without the loop measurements, from the
    same starting state, to give the measurements' cost."""
    own_view = view is None and ens.precision == F32_TWO_ROW
    if own_view:
        view = ens.like(precision=F64)
    try:
        start_sweep = ens.sweep_index
        saved = None
        if time_sweeps_alone:
            saved = ens.like()
            ens.copy_to(saved)
            ens.synchronize()
            t0 = time.perf_counter()
            ens.measured_sweeps(proposal_angle, n_blocks * sweeps_per_block, 1, generator_mode)
            sweep_secs = time.perf_counter() - t0
            saved.copy_to(ens)
            ens.sweep_index = start_sweep
        ens.synchronize()
        t0 = time.perf_counter()
        plaq, wil, pol = ens.measured_run(proposal_angle, n_blocks, sweeps_per_block, rmax, tmax,
                                          polyakov_direction, generator_mode, view=view)
        secs = time.perf_counter() - t0
        if saved is not None:
            saved.close()
    finally:
        if own_view:
            view.close()
    links = int(sum(np.prod(e) * 4 for e in ens.extents))
    return MeasuredRunResult([tuple(e) for e in ens.extents], ens.precision, sweeps_per_block, plaq,
                             wil, pol, secs, sweep_secs if time_sweeps_alone else float("nan"),
                             links * n_blocks * sweeps_per_block)


@dataclass
class PrecisionComparison:
    fp32: MeasuredRunResult
    fp64: MeasuredRunResult
    plaquette_mean_fp32: float
    plaquette_mean_fp64: float
    plaquette_error: float             # |mean FP32 - mean FP64|
    plaquette_combined_sigma: float    # combined standard error of the two means
    first_sweep_plaquette_error: float # max over chains after the first sweep (same field, same streams)
    wilson_max_error: float            # max |W_32 - W_64| over blocks, chains, planes, R, T
    polyakov_max_error: float


def fp32_vs_fp64_run(start: Ensemble, n_blocks: int, sweeps_per_block: int = 10,
                     proposal_angle: float = 0.3, generator_mode: str = "ordered",
                     max_lag: int = 20) -> PrecisionComparison:
    """The cadence run twice from the binary64 field of ``start`` (its seeds
    and sweep index): in two-row binary32 and in binary64.  Both runs start
    from the same links (the binary32 copy rounds them), draw from the same
    per-link streams and measure the same observables; the comparison states
    the binary32 run's error against the binary64 one.  Trajectories of the
    two runs separate after a few sweeps (Metropolis decisions near the
    threshold flip), so the plaquette is compared as run means with their
    combined standard error; the first sweep is compared directly."""
    sweep = start.sweep_index
    with start.like(precision=F32_TWO_ROW) as f32, start.like(precision=F64) as f64, \
            start.like(precision=F64) as view:
        start.convert_to(f32)
        f32.sweep_index = sweep
        start.copy_to(f64)
        f64.sweep_index = sweep
        r32 = su3_measured_run(f32, n_blocks, sweeps_per_block, proposal_angle, generator_mode, view=view)
        r64 = su3_measured_run(f64, n_blocks, sweeps_per_block, proposal_angle, generator_mode)

    def mean_err(series):
        flat = series.mean(1)
        lag = max(1, min(max_lag, len(flat) - 1))
        d = diagnostics(flat, lag)[0]
        return float(flat.mean()), float(d.standard_error)

    m32, e32 = mean_err(r32.plaquette)
    m64, e64 = mean_err(r64.plaquette)
    return PrecisionComparison(
        r32, r64, m32, m64, abs(m32 - m64), float(np.hypot(e32, e64)),
        float(np.max(np.abs(r32.plaquette[0] - r64.plaquette[0]))),
        float(np.max(np.abs(r32.wilson - r64.wilson))),
        float(np.max(np.abs(r32.polyakov - r64.polyakov))))


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
    prepare_seconds: float = 0.0      # building the measurement graph, once
    link_updates: int = 0
    sweep_layout: dict = field(default_factory=dict)   # the handle tuner's choice
    sweep_path: str = ""


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
    # chains are listed group by group, so each group's chains are consecutive
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
        blocked_groups = sorted(subs)
        # slice offsets: every chain's N3 time slices, chain by chain (the
        # smeared handle), and per blocked group in the blocked outputs
        slice_at = np.concatenate([[0], np.cumsum([e[3] for e in extents])]).astype(int)
        blocked_at, k = {}, 0
        for gi in blocked_groups:
            blocked_at[gi] = k
            k += sum(extents[c][3] for c in per_group[gi])
        levels_sorted = sorted(stout_levels)
        plan_blocked = [(subs[gi], coarse[gi], per_group[gi][0]) for gi in blocked_groups]
        try:
            # the measurement graph, built once before the first measurement
            t0 = time.perf_counter()
            ens.glueball_prepare(sm, levels_sorted, rho, plan_blocked)
            res.prepare_seconds = time.perf_counter() - t0
            t0 = time.perf_counter()
            ens.metropolis_sweeps(proposal_angle, thermalization)
            ens.synchronize()
            res.sweep_seconds += time.perf_counter() - t0
            res.sweep_layout = ens.sweep_layout
            res.sweep_path = ens.sweep_path
            for _ in range(measurements):
                t0 = time.perf_counter()
                ens.metropolis_sweeps(proposal_angle, sweeps_between_measurements)
                ens.synchronize()
                t1 = time.perf_counter()
                res.sweep_seconds += t1 - t0
                # one captured graph: the levels continue from the previous
                # count (0, 5, 10 costs 10 levels, not 15; the same links as
                # smearing from scratch), operators after each count, the
                # blockable groups blocked and measured
                plaq, rect, bplaq, brect = ens.glueball_measure(sm, levels_sorted, rho, plan_blocked)
                # a group's chains are consecutive, so its time slices form one
                # (chains, N3) block of every output row
                for li, levels in enumerate(levels_sorted):
                    for gi, chains in enumerate(per_group):
                        nt, a = extents[chains[0]][3], slice_at[chains[0]]
                        n = len(chains) * nt
                        samples.setdefault((gi, levels, False), []).append(
                            (plaq[li, a:a + n].reshape(len(chains), nt).copy(),
                             rect[li, a:a + n].reshape(len(chains), nt).copy()))
                        if gi in subs:
                            k0 = blocked_at[gi]
                            samples.setdefault((gi, levels, True), []).append(
                                (bplaq[li, k0:k0 + n].reshape(len(chains), nt).copy(),
                                 brect[li, k0:k0 + n].reshape(len(chains), nt).copy()))
                res.measure_seconds += time.perf_counter() - t1
        finally:
            for h in list(coarse.values()) + list(subs.values()) + [sm]:
                h.close()
        res.link_updates = int(sum(np.prod(e) * 4 for e in extents)) * (
            thermalization + measurements * sweeps_between_measurements)
    for (gi, levels, blocked), blocks in sorted(samples.items()):
        # rows: measurement by measurement, chains in order within each
        p = np.concatenate([blk[0] for blk in blocks])
        r = np.concatenate([blk[1] for blk in blocks])
        nt = p.shape[1]
        reps = G.jackknife_replicas(p)
        end = min(4, nt // 2)
        cov = G.jackknife_covariance(reps, 1, end) if len(reps) > end else np.zeros((0, 0))
        res.surfaces.append(SurfaceResult(
            tuple(groups[gi][1]) if not blocked else G.blocked_extents(groups[gi][1]),
            levels, blocked, p, r, G.connected_from_samples(p), G.connected_from_samples(r),
            reps, cov))
    return res
