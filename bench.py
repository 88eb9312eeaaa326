#!/usr/bin/env python3
"""Throughput of the B200 lattice gauge engine on its headline workload.

Workload (one GPU): SU(3) Wilson action, periodic 32^4, beta = 6.0, FP64
links, Haar hot start, single-generator Metropolis with the reference's
eight ordered generator hits per link visit and the paired angle grid of
half width 0.3, updated over an even/odd checkerboard.  One step = one full
sweep of every link followed by an average-plaquette measurement.  The
lattice (604 MB) is larger than the 126 MB L2, so no flush is needed between
steps.  ``value`` is link updates/s (one link visit = eight proposals) over
all GPUs; the plaquette series of the timed steps gives the plaquette ESS/s
through the reference's autocorrelation estimator.

``--impl reference`` times the reference's own algorithm (the lexicographic
single-stream Metropolis sweep with twelve-plaquette action differences,
restated in C in oracle/) on the host cores; see oracle/or_threads.c.

Launch: ``python bench.py --gpus N --steps K --warmup W`` (torchrun for N > 1:
independent replicas, one lattice per GPU, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "yang-mills_b200"))

METRIC = "SU(3) link updates/s and plaquette ESS/s, learned vs plain Metropolis"
UNIT = "link updates/s"
EXTENTS = [32, 32, 32, 32]
BETA = 6.0
ANGLE = 0.3
THERMALIZATION = 400                  # 3/4 at angle 1.0 (fast relaxation), 1/4 at ANGLE
THERMALIZATION_ANGLE = 1.0
MASTER_SEED = 0x2C02198105010002
LINK_BYTES = 144                      # FP64 3x3 complex
LINKS_PER_UPDATE = 9                  # 8 link reads + 1 write per checkerboard update
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--thermalization", type=int, default=THERMALIZATION)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic_per_launch():
    """DRAM bytes per k_su3_metropolis launch from the committed ncu summary,
    scaled to a 32^4 launch (None when no summary exists)."""
    path = os.path.join(ROOT, "profiles", "su3_metropolis_f64.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_32^4_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"ym_clocks_{os.getpid()}.csv")
        self.first = self.last = 0

    def _rows(self):
        try:
            with open(self.path) as fh:
                return [ln for ln in fh.read().splitlines() if ln.count(",") >= 8]
        except OSError:
            return []

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def wait_first(self, timeout=5.0):
        """Block until nvidia-smi has written a sample, so that every later
        sample falls inside the region that follows."""
        end = time.time() + timeout
        while self.proc and time.time() < end and not self._rows():
            time.sleep(0.02)
        self.first = len(self._rows())

    def mark_end(self):
        self.last = len(self._rows())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [[p.strip() for p in ln.split(",")] for ln in self._rows()]
        inside = rows[self.first:self.last]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"],
                    "samples": 0}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [num(r[1]) for r in inside if num(r[1]) is not None]
        mx = [num(r[2]) for r in inside if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in inside for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(inside), "interval_ms": 100}


def cpu_baseline(seconds_target=12.0):
    """The reference algorithm (oracle port) on all host threads, 16^4
    lattices (the reference's 2^18-link cap), per link update."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    ext = [16, 16, 16, 16]
    t, n = O.bench_su3_reference(ext, BETA, ANGLE, MASTER_SEED, 1, 32)
    per_thread = max(32, int(seconds_target * n / max(t, 1e-9)))
    secs, done = O.bench_su3_reference(ext, BETA, ANGLE, MASTER_SEED, threads, per_thread)
    return {"value": done / secs, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{threads} threads x {per_thread} link visits (8 ordered hits each) of an "
                      f"independent cold 16^4 lattice, beta={BETA}, angle={ANGLE}, "
                      f"{secs:.1f} s wall"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    ext = [16, 16, 16, 16]
    t, n = O.bench_su3_reference(ext, BETA, ANGLE, MASTER_SEED, 1, 32)
    step_target = 1.5
    per_thread = max(16, int(step_target * n / max(t, 1e-9)))
    for w in range(args.warmup):
        O.bench_su3_reference(ext, BETA, ANGLE, MASTER_SEED + w, threads, per_thread)
    total_s, total_n = 0.0, 0
    for k in range(args.steps):
        secs, done = O.bench_su3_reference(ext, BETA, ANGLE, MASTER_SEED + 1000 + k, threads,
                                           per_thread)
        total_s += secs
        total_n += done
    value = total_n / total_s
    sample = (f"each step: {threads} threads x {per_thread} link visits of independent cold 16^4 "
              f"lattices (reference algorithm restated in C, not the reference binary)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "SU(3) Metropolis, beta=6.0, 8 ordered hits per link visit",
                   "lattice": "16^4 per thread (reference cap 2^18 links)",
                   "parallelism": f"{threads} independent chains, one per host thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    import numpy as np
    import torch
    import torch.distributed as dist
    import ymgpu
    from ymgpu.su2_ensemble import diagnostics

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    seed = ymgpu.su3_ensemble.derive_su3_chain_seed(MASTER_SEED, rank)
    volume = int(np.prod(EXTENTS))
    links = 4 * volume
    peak, peak_kind = measured_peaks()

    def max_over_ranks(x):
        if world > 1:
            t = torch.tensor([x], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    def run_leg(precision, link_bytes, sampler_clocks=False):
        """Thermalise, then time args.steps steps (sweep [+ reunitarise] +
        plaquette) with CUDA events on the handle's stream."""
        ens = ymgpu.Ensemble([EXTENTS], BETA, seed, precision=precision,
                             lift_reference_caps=True, device=local)
        ens.hot_start()
        wide = (3 * args.thermalization) // 4
        ens.metropolis_sweeps(THERMALIZATION_ANGLE, wide)
        ens.metropolis_sweeps(ANGLE, args.thermalization - wide)
        for _ in range(args.warmup):
            ens.metropolis_sweeps(ANGLE, 1)
            ens.average_plaquette()
        ens.synchronize()
        stream = torch.cuda.ExternalStream(ens.stream(), device=local)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0, a0 = ens.accounting()
        plaq = []
        ens.profile(True)
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if sampler_clocks else None
        if sampler:
            sampler.__enter__()
            sampler.wait_first()
        start.record(stream)
        for _ in range(args.steps):
            ens.metropolis_sweeps(ANGLE, 1)     # two-row handles reunitarise inside the sweep
            plaq.append(float(ens.average_plaquette()[0]))
        stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
        if sampler:
            sampler.mark_end()
            sampler.__exit__(None, None, None)
        barrier()
        ms = max_over_ranks(start.elapsed_time(stop))
        sweep_ms, sweep_launches = ens.profile_read("su3_metropolis")
        ens.profile(False)
        p1, a1 = ens.accounting()
        # plaquette ESS/s through the reference estimator (su2_ensemble.rs:375-463)
        max_lag = max(1, min(len(plaq) // 4, 50))
        diag, _ = diagnostics(np.array(plaq), max_lag)
        # roofline of the dominant kernel (one checkerboard sub-sweep launch)
        launch_s = sweep_ms * 1e-3 / max(1, sweep_launches)
        achieved = (volume // 2) * LINKS_PER_UPDATE * link_bytes / launch_s / 1e9
        return ens, {
            "ms": ms, "value": world * links * args.steps / (ms * 1e-3),
            "plaq": plaq, "diag": diag,
            "ess_per_s": world * diag.effective_sample_size / (ms * 1e-3),
            "acceptance": float((a1 - a0)[0]) / float((p1 - p0)[0]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "launch_ms": launch_s * 1e3, "kernel_share_of_step": sweep_ms / ms,
                         "bytes_per_launch": (volume // 2) * LINKS_PER_UPDATE * link_bytes},
            "clocks": sampler.summary() if sampler else None,
        }

    # binary32 two-row leg (BASELINE configs[2] link algebra), reported beside
    f32_ens, f32 = run_leg(ymgpu.F32_TWO_ROW, 48)
    f32_ens.close()
    ens, leg = run_leg(ymgpu.F64, LINK_BYTES, sampler_clocks=True)
    ms, plaq, diag = leg["ms"], leg["plaq"], leg["diag"]
    step_ms = ms / args.steps
    value = leg["value"]
    ess_per_s = leg["ess_per_s"]
    clocks = leg["clocks"]
    roofline = dict(leg["roofline"])
    roofline.update({"traffic": ncu_traffic_per_launch(),
                     "kernel": "k_su3_metropolis (one checkerboard sub-sweep)"})

    # end to end through the C ABI with host buffers: upload the lattice from
    # pinned host memory, sweep, measure, download the lattice
    host = torch.empty(links * 18, dtype=torch.float64, pin_memory=True)
    host_np = host.numpy().view(np.complex128).reshape(links, 3, 3)
    ens.download(0, host_np)
    e2e_steps = max(3, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ens.upload(0, host_np)
        ens.metropolis_sweeps(ANGLE, 1)
        ens.average_plaquette()
        ens.download(0, host_np)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0)
    e2e = {"value": world * links * e2e_steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": links * LINK_BYTES,
           "d2h_bytes_per_step": links * LINK_BYTES + 8,
           "path": "ym_ensemble_upload -> ym_su3_metropolis_sweeps -> ym_average_plaquette "
                   "-> ym_ensemble_download (pinned host lattice in the reference layout)"}
    ens.close()

    if rank == 0:
        cpu = None if (args.no_cpu_baseline or world > 1) else cpu_baseline()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "SU(3) 32^4 beta=6.0 plain FP64 Metropolis (configs[2] "
                                   "geometry), 8 ordered hits/link, angle 0.3, Haar hot start "
                                   f"+ {args.thermalization} untimed thermalization sweeps "
                                   "(3/4 at angle 1.0, 1/4 at 0.3)",
                       "lattice": "32^4", "global_batch": world, "parallelism": f"replicas x{world}",
                       "l2": "inputs 604 MB > 126 MB L2 (no flush)",
                       "step": "1 checkerboard sweep + average plaquette"},
            "plaquette_mean": float(np.mean(plaq)),
            "plaquette_ess_per_s": ess_per_s,
            "plaquette_tau_int": diag.integrated_autocorrelation_time,
            "acceptance": leg["acceptance"],
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(args.steps * 11),
            "clocks": clocks,
            "fp32_two_row": {
                "value": f32["value"], "unit": UNIT, "dtype": "f32 links, f64 dS/accept/plaquette",
                "ms_per_step": f32["ms"] / args.steps,
                "step": "1 checkerboard sweep + FP64 reunitarisation + average plaquette",
                "plaquette_mean": float(np.mean(f32["plaq"])),
                "plaquette_minus_f64": float(np.mean(f32["plaq"]) - np.mean(plaq)),
                "plaquette_ess_per_s": f32["ess_per_s"], "acceptance": f32["acceptance"],
                "roofline": f32["roofline"]},
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
