#!/usr/bin/env python3
"""Throughput of the B200 lattice gauge engine on its headline workload.

Workload (one GPU): SU(3) Wilson action, periodic 32^4, beta = 6.0, FP64
links, Haar hot start thermalised by wide-angle sweeps, single-generator
Metropolis with the reference's eight ordered generator hits per link visit
and the paired angle grid of half width 0.3, updated over an even/odd
checkerboard.  One step = one full sweep of every link followed by an
average-plaquette measurement.  The lattice (604 MB) is larger than the
126 MB L2, so no flush is needed between steps.  ``value`` is link updates/s
(one link visit = eight proposals) over all GPUs.

Beside it: the same FP64 steps in the fast form (``fp64_fast``: fused
multiply-adds and Horner rotations, with its distance from the exact form
after ten sweeps), the same steps with two-row binary32 links (``fp32_two_row``),
with the learned proposal (``learned``: its network trained on the GPU on
2000 configurations of the plain sampler), and the plaquette ESS/s of plain
FP64, plain FP32 (half width 0.3 and, as a control, the widest the
reference admits, 1.0) and learned FP32 sampling at the learned-proposal geometry
(16 chains of 16^4 in one handle, the total volume of 32^4), each judged by
the reference's autocorrelation estimator (su2_ensemble.rs:375-463) on
per-chain plaquette series.

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
THERMALIZATION = 1500                 # wide-angle sweeps from the hot start
THERMALIZATION_ANGLE = 1.0            # the plaquette relaxes fastest at wide angles
ESS_CHAINS, ESS_EXTENTS = 16, [16, 16, 16, 16]
ESS_SWEEPS = 3000                     # measured sweeps per sampler (one plaquette each)
TRAIN_STEPS = 2000                    # configurations the plain sampler generates for training
TRAIN_LR = 3e-3
LOOP_BLOCKS = 10                      # loop measurements per run of the loop cadence
LOOP_EVERY = 10                       # sweeps between Wilson / Polyakov measurements
FAST_CHECK_SWEEPS = 10                # sweeps per form when the fast form is compared with the exact one
MASTER_SEED = 0x2C02198105010002
LINK_BYTES = 144                      # FP64 3x3 complex
E2E_LATTICES = 4                      # independent lattices in flight end to end (upload, sweep, download)
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
    ap.add_argument("--ess-sweeps", type=int, default=ESS_SWEEPS)
    ap.add_argument("--train-steps", type=int, default=TRAIN_STEPS)
    ap.add_argument("--loop-blocks", type=int, default=LOOP_BLOCKS)
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
    """DRAM bytes per k_su3_metropolis_ring launch from the committed ncu summary,
    scaled to a 32^4 launch (None when no summary exists)."""
    path = os.path.join(ROOT, "profiles", "su3_metropolis_32x4_fp64.md")
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

    INTERVAL_MS = 10

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
                 "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)], stdout=self.fh,
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

    def summary(self, whole=False):
        """Samples inside the timed region (whole: every sample the sampler
        took, from before the warm-up steps to after the timed ones)."""
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [[p.strip() for p in ln.split(",")] for ln in self._rows()]
        inside = rows if whole else rows[self.first:self.last]
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
                "samples": len(inside), "interval_ms": self.INTERVAL_MS}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


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
            "cpu_model": cpu_model(),
            "sample": f"{threads} threads x {per_thread} link visits (8 ordered hits each) of an "
                      f"independent cold 16^4 lattice, beta={BETA}, angle={ANGLE}, "
                      f"{secs:.1f} s wall; the lattices start cold (the reference's run_chain "
                      "start), which does not change the cost of a visit: the reference's visit "
                      "does the same twelve-plaquette products, exponential and checks whatever "
                      "the link values"}


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
              f"lattices (reference algorithm restated in C, not the reference binary; a cold "
              f"start does not change the cost of a visit, whose products and checks are the "
              f"same whatever the link values)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "SU(3) Metropolis, beta=6.0, 8 ordered hits per link visit",
                   "lattice": "16^4 per thread (reference cap 2^18 links)",
                   "parallelism": f"{threads} independent chains, one per host thread"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "cpu_model": cpu_model(), "sample": sample},
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
    import ymgpu
    from ymgpu.replicas import Replicas
    from ymgpu.su2_ensemble import diagnostics
    from ymgpu.su3_ensemble import derive_su3_chain_seed

    torch.cuda.set_device(local)
    # one process per GPU, replicas only: barrier, slowest-rank timing, rank-0 output
    rep = Replicas(backend="nccl", timeout_s=120, device=torch.device("cuda", local))
    barrier = rep.barrier
    max_over_ranks = rep.max_over_ranks
    seed = rep.chain_seed(MASTER_SEED)
    volume = int(np.prod(EXTENTS))
    links = 4 * volume
    peak, peak_kind = measured_peaks()

    def timed_leg(ens, step, link_bytes, kernel, measured, sampler_clocks=False):
        """The run_chain cadence of one leg: W warm-up steps, then args.steps
        steps (one sweep, then the average plaquette of the swept lattice),
        timed with CUDA events on the handle's stream.  measured(n) runs n
        steps through the library's measured-sweeps entry point (one captured
        graph per step, the plaquette of every step stored on the device and
        read back once) and returns the plaquette series.  The last n_prof
        steps of the timed region are issued one launch at a time with an
        event pair around each launch (step() = one sweep, then
        average_plaquette): they give the dominant kernel's per-launch time
        and its share of a step, inside the timed region.  With
        sampler_clocks, nvidia-smi samples every 10 ms from before the
        warm-up to after the timed steps: "clocks" summarises the samples
        inside the timed region, "clocks_leg" all of them."""
        sampler = ClockSampler(local) if sampler_clocks else None
        if sampler:
            sampler.__enter__()
            sampler.wait_first()
        measured(args.warmup)
        step()
        ens.average_plaquette()
        ens.synchronize()
        n_prof = max(1, min(20, args.steps // 4))
        n_graph = args.steps - n_prof
        stream = torch.cuda.ExternalStream(ens.stream(), device=local)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        pa, pb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0, a0 = ens.accounting()
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.wait_first()
        start.record(stream)
        series = measured(n_graph) if n_graph > 0 else np.zeros((0, 1))
        plaq = [float(v) for v in np.asarray(series)[:, 0]]
        ens.profile(True)
        pa.record(stream)
        for _ in range(n_prof):
            step()
            plaq.append(float(ens.average_plaquette()[0]))
        pb.record(stream)
        stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
        if sampler:
            sampler.mark_end()
            sampler.__exit__(None, None, None)
        barrier()
        ms = max_over_ranks(start.elapsed_time(stop))
        k_ms, k_launches = ens.profile_read(kernel)
        ens.profile(False)
        p1, a1 = ens.accounting()
        launch_s = k_ms * 1e-3 / max(1, k_launches)
        bytes_per_launch = (volume // 2) * LINKS_PER_UPDATE * link_bytes
        achieved = bytes_per_launch / launch_s / 1e9
        return {
            "ms": ms, "value": world * links * args.steps / (ms * 1e-3), "plaq": plaq,
            "acceptance": float((a1 - a0)[0]) / float((p1 - p0)[0]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "launch_ms": launch_s * 1e3,
                         "kernel_share_of_step": k_ms / max(1e-9, pa.elapsed_time(pb)),
                         "bytes_per_launch": bytes_per_launch,
                         "per_launch_steps": n_prof,
                         "note": f"per-launch events over the last {n_prof} of the {args.steps} timed steps, "
                                 "issued launch by launch (the others through the measured-sweeps graphs)"},
            "clocks": sampler.summary() if sampler else None,
            "clocks_leg": sampler.summary(whole=True) if sampler else None,
        }

    # one thermalised 32^4 lattice (two-row binary32; wide-angle sweeps relax
    # the plaquette fastest), shared by all legs
    t32 = ymgpu.Ensemble([EXTENTS], BETA, seed, precision=ymgpu.F32_TWO_ROW,
                         lift_reference_caps=True, device=local)
    t32.hot_start()
    t32.metropolis_sweeps(THERMALIZATION_ANGLE, args.thermalization, "uniform")

    # learned proposal: network trained on configurations of the plain
    # sampler at the learned-proposal geometry (16 x 16^4)
    ess_seeds = [derive_su3_chain_seed(MASTER_SEED ^ 0x16, rank * ESS_CHAINS + i)
                 for i in range(ESS_CHAINS)]
    e16 = ymgpu.Ensemble([ESS_EXTENTS] * ESS_CHAINS, BETA, ess_seeds, precision=ymgpu.F32_TWO_ROW,
                         lift_reference_caps=True, device=local)
    e16.hot_start()
    e16.metropolis_sweeps(THERMALIZATION_ANGLE, args.thermalization, "uniform")
    model = ymgpu.ProposalModel(device=local, initial_scale=ANGLE)
    e16.synchronize()
    t0 = time.perf_counter()
    train_hist = model.train(e16, args.train_steps, sweeps_per_step=1, plain_angle=ANGLE, lr=TRAIN_LR)
    train_s = time.perf_counter() - t0
    f_rec, _, _ = ymgpu.learned.records(e16, 0, 0)
    p_gen, s_half = ymgpu.learned.proposal(model.forward(f_rec))

    # FP32 plain leg (ordered generators, half width 0.3)
    f32 = timed_leg(t32, lambda: t32.metropolis_sweeps(ANGLE, 1), 48, "su3_metropolis",
                    lambda n: t32.measured_sweeps(ANGLE, n, 1, "ordered"))
    # learned leg from the same starting lattice
    tl = t32.like()
    t32.copy_to(tl)
    lrn = timed_leg(tl, lambda: model.sweeps(tl, 1), 48, "learned",
                    lambda n: model.measured_sweeps(tl, n, 1))
    tl.close()
    # FP64 headline leg
    ens = t32.like(precision=ymgpu.F64)
    t32.convert_to(ens)
    t32.close()
    leg = timed_leg(ens, lambda: ens.metropolis_sweeps(ANGLE, 1), LINK_BYTES, "su3_metropolis",
                    lambda n: ens.measured_sweeps(ANGLE, n, 1, "ordered"), sampler_clocks=True)
    ms, plaq = leg["ms"], leg["plaq"]
    roofline = dict(leg["roofline"])
    roofline.update({"traffic": ncu_traffic_per_launch(),
                     "kernel": "k_su3_metropolis_ring (ordered hits; one checkerboard sub-sweep)"})

    # the same FP64 step in the fast form (fused multiply-adds, Horner
    # rotations; ym_ensemble_set_fast_sweeps) from a copy of the same lattice,
    # then its distance from the exact form: two copies of the lattice after
    # that leg, ten sweeps each from the same sweep index, exact and fast
    fast_src = ens.like()
    ens.copy_to(fast_src)
    fast_src.sweep_index = ens.sweep_index
    fast_src.fast_sweeps = True
    fleg = timed_leg(fast_src, lambda: fast_src.metropolis_sweeps(ANGLE, 1), LINK_BYTES, "su3_metropolis",
                     lambda n: fast_src.measured_sweeps(ANGLE, n, 1, "ordered"))
    pair = []
    for fast in (False, True):
        c = fast_src.like()
        fast_src.copy_to(c)
        c.sweep_index = fast_src.sweep_index
        c.fast_sweeps = fast
        c.reset_accounting()
        c.metropolis_sweeps(ANGLE, FAST_CHECK_SWEEPS, "ordered")
        pair.append((c.download(0), int(c.accounting()[1][0]), float(c.average_plaquette()[0])))
        c.close()
    fast_src.close()
    fast_err = {
        "sweeps": FAST_CHECK_SWEEPS, "lattice": "32^4, the bench lattice after the fast leg",
        "max_abs_link_entry_difference": float(np.max(np.abs(pair[0][0] - pair[1][0]))),
        "accepts_exact": pair[0][1], "accepts_fast": pair[1][1],
        "plaquette_difference": pair[1][2] - pair[0][2]}
    del pair

    # spatial stout smearing of a 32^4 FP64 lattice (rho 0.1), each level
    # timed by its CUDA-event pair; compulsory traffic per level: every link
    # of every site read once and written once.  The reference's smearing
    # checks every link against SU(3) to 5e-12, so the lattice is an FP64
    # Haar hot start swept in FP64 (the thermalised one above came from
    # binary32 storage).
    src = ens.like()
    src.hot_start()
    src.metropolis_sweeps(1.0, 20, "uniform")
    sm = src.like()
    src.stout_smear_into(sm, 0.1, 1, lift_level_cap=True)
    sm.profile(True)
    src.stout_smear_into(sm, 0.1, 4, lift_level_cap=True)
    st_ms, st_n = sm.profile_read("stout")
    sm.profile(False)
    sm.close()
    src.close()
    st_s = st_ms * 1e-3 / max(1, st_n)
    st_bytes = volume * 8 * LINK_BYTES
    stout = {"ms_per_level": st_s * 1e3, "levels_timed": st_n, "bytes_per_level": st_bytes,
             "roofline": {"bound": "hbm", "achieved": st_bytes / st_s / 1e9, "peak": peak,
                          "unit": "GB/s", "frac": st_bytes / st_s / 1e9 / peak,
                          "peak_source": f"{peak_kind} hbm_gbs",
                          "kernel": "k_stout_level (staples, Q, Cayley-Hamilton exponential "
                                    "with the reference's checks, per spatial link)"}}

    # observables of the thermalised 32^4 FP64 lattice, each call timed by the
    # handle's CUDA-event pair around its kernels: Wilson loops R x T <= 4 x 4
    # in all six planes, the Polyakov loop along direction 3, the A1++
    # operator basis (spatial plaquettes and 2x1 rectangles per timeslice).
    # Compulsory traffic: each link the observable reads, once (4V links for
    # the loops, V for the Polyakov loop, 3V spatial links for the operators).
    def obs_leg(kernel, call, n_links, reps=3):
        call()
        ens.profile(True)
        for _ in range(reps):
            call()
        o_ms, o_n = ens.profile_read(kernel)
        ens.profile(False)
        o_s = o_ms * 1e-3 / max(1, o_n)
        o_bytes = volume * n_links * LINK_BYTES
        return {"ms": o_s * 1e3, "calls_timed": o_n, "compulsory_bytes": o_bytes,
                "achieved_gbs": o_bytes / o_s / 1e9, "frac": o_bytes / o_s / 1e9 / peak}

    wilson = obs_leg("aux", lambda: ens.wilson_loops(4, 4), 4)
    # its arithmetic: per site and plane 38 3x3 complex products (D_T, A_R,
    # P_{R,T}, Q_{R,T} for R, T <= 4), each 9 entries x 3 complex fma =
    # 216 flops, so 8,208 flops (the 16 traces not counted); the ratio is to
    # the B200's nominal 37 TFLOP/s FP64 (no measured FP64 peak exists here)
    w_flops = volume * 6 * 38 * 216
    wilson.update({"fp64_tflops": w_flops / (wilson["ms"] * 1e-3) / 1e12,
                   "fp64_frac_of_nominal_37": w_flops / (wilson["ms"] * 1e-3) / 37e12})
    observables = {
        "wilson_loops_4x4_all_planes": wilson,
        "polyakov_loop_dir3": obs_leg("aux", lambda: ens.polyakov_loops(3), 1),
        "a1pp_operator_basis": obs_leg("operators", ens.scalar_operator_basis, 3),
        "peak_gbs": peak, "peak_source": f"{peak_kind} hbm_gbs",
        "note": "per call on the 32^4 FP64 lattice; achieved = compulsory bytes / CUDA-event time"}

    # the loop-measurement cadence (two-row FP32 sweeps with FP64
    # reunitarisation and plaquette every sweep; Wilson loops R x T <= 4 x 4
    # and Polyakov loops every LOOP_EVERY sweeps, one captured graph per
    # block) at 32^4 and 24^3 x 48, each against an FP64 run of the same
    # length from the same field, seeds and sweep indices
    from ymgpu.pipelines import fp32_vs_fp64_run

    def loop_cadence(start):
        c = fp32_vs_fp64_run(start, n_blocks=args.loop_blocks, sweeps_per_block=LOOP_EVERY,
                             proposal_angle=ANGLE, generator_mode="ordered")
        out = {}
        for name, r in (("fp32_two_row", c.fp32), ("fp64", c.fp64)):
            out[name] = {"link_updates_per_s": world * r.link_updates_per_s, "seconds": r.seconds,
                         "sweep_only_seconds": r.sweep_seconds,
                         "loop_measurement_seconds": r.loop_measurement_seconds,
                         "loop_measurement_share": r.loop_measurement_seconds / r.seconds,
                         "plaquette_mean": float(r.plaquette.mean()),
                         "wilson_1x1_mean": float(r.wilson[:, :, :, 0, 0].mean()),
                         "wilson_4x4_mean": float(r.wilson[:, :, :, 3, 3].mean()),
                         "polyakov_abs_mean": float(np.abs(r.polyakov).mean())}
        out["error_fp32_vs_fp64"] = {
            "plaquette_mean_difference": c.plaquette_error,
            "plaquette_combined_standard_error": c.plaquette_combined_sigma,
            "plaquette_difference_in_sigma": c.plaquette_error / c.plaquette_combined_sigma,
            "first_sweep_plaquette_difference": c.first_sweep_plaquette_error,
            "wilson_max_abs_difference": c.wilson_max_error,
            "polyakov_max_abs_difference": c.polyakov_max_error,
            "note": "trajectories separate after a few sweeps (decisions near the threshold "
                    "flip), so the run means are compared with their combined standard error "
                    "(reference estimator on the per-sweep series); the first sweep, from the "
                    "same field and streams, directly"}
        out["schedule"] = (f"{args.loop_blocks} blocks x {LOOP_EVERY} sweeps, half width {ANGLE}, "
                           "8 ordered hits; plaquette every sweep, loops every block")
        return out

    cad_start = ens.like()
    ens.copy_to(cad_start)
    cad_start.sweep_index = ens.sweep_index
    loop_runs = {"32^4": loop_cadence(cad_start)}
    cad_start.close()
    e48 = ymgpu.Ensemble([[24, 24, 24, 48]], BETA, seed, precision=ymgpu.F32_TWO_ROW,
                         lift_reference_caps=True, device=local)
    e48.hot_start()
    e48.metropolis_sweeps(THERMALIZATION_ANGLE, args.thermalization, "uniform")
    s48 = e48.like(precision=ymgpu.F64)
    e48.convert_to(s48)
    s48.sweep_index = e48.sweep_index
    e48.close()
    loop_runs["24^3x48"] = loop_cadence(s48)
    s48.close()

    # plaquette ESS/s of the three samplers at 16 x 16^4 from one equilibrated state
    def ess_leg(e, run):
        e.synchronize()
        t = time.perf_counter()
        series = run()
        secs = time.perf_counter() - t
        lag = max(1, min(500, series.shape[0] // 4))
        diags = [diagnostics(series[:, c], lag)[0] for c in range(series.shape[1])]
        ess = float(sum(d.effective_sample_size for d in diags))
        means = series.mean(0)
        return {"plaquette_ess_per_s": world * ess / secs, "seconds": secs,
                "tau_int": float(np.mean([d.integrated_autocorrelation_time for d in diags])),
                "plaquette_mean": float(means.mean()),
                "plaquette_error": float(means.std(ddof=1) / np.sqrt(len(means))),
                "link_updates_per_s": world * 4 * int(np.prod(ESS_EXTENTS)) * ESS_CHAINS *
                                      series.shape[0] / secs}

    e64 = e16.like(precision=ymgpu.F64)
    e16.convert_to(e64)
    e32p = e16.like()
    e16.copy_to(e32p)
    e32w = e16.like()
    e16.copy_to(e32w)
    # matched control: plain uniform-generator Metropolis at the constant half
    # width the trained network settles at (its mean over the lattice's
    # links), past the reference's cap of 1.0 behind the handle's explicit lift
    s_bar = float(np.mean(s_half))
    e32c = e16.like()
    e16.copy_to(e32c)
    e32c.lift_angle_cap(True)
    n = args.ess_sweeps
    ess_f64 = ess_leg(e64, lambda: e64.measured_sweeps(ANGLE, n, 1, "ordered"))
    ess_f32 = ess_leg(e32p, lambda: e32p.measured_sweeps(ANGLE, n, 1, "uniform"))
    ess_f32w = ess_leg(e32w, lambda: e32w.measured_sweeps(1.0, n, 1, "uniform"))
    ess_f32c = ess_leg(e32c, lambda: e32c.measured_sweeps(s_bar, n, 1, "uniform"))
    ess_f32c["half_width"] = s_bar
    ess_lrn = ess_leg(e16, lambda: model.measured_sweeps(e16, n))
    for e in (e64, e32p, e32w, e32c, e16):
        e.close()
    model.close()
    sig = lambda a, b: abs(a["plaquette_mean"] - b["plaquette_mean"]) / np.hypot(
        a["plaquette_error"], b["plaquette_error"])

    # the other configurations of the path, each short: throughput and
    # plaquette ESS/s through the same estimator
    def other_configs():
        out = {}
        from ymgpu.su2_ensemble import derive_chain_seed
        # SU(2) 10^4 beta=2.3: 1 Kennedy-Pendleton heat-bath + 3 overrelaxation per sweep
        e2 = ymgpu.Ensemble([[10, 10, 10, 10]], 2.3, derive_chain_seed(0x2B00201211160101, rank),
                            group=ymgpu.SU2, device=local)
        e2.set_identity()
        e2.markov_sweeps(200, 3, sampler="kennedy-pendleton")
        e2.synchronize()
        t = time.perf_counter()
        series = e2.su2_measured_sweeps(500, 1, 3, sampler="kennedy-pendleton")[:, 0]
        secs = time.perf_counter() - t
        # per-launch device time of the two update kernels (one launch = one
        # parity and direction: 5,000 links), 20 more sweeps under the events
        e2.profile(True)
        e2.markov_sweeps(20, 3, sampler="kennedy-pendleton")
        hb_ms, hb_n = e2.profile_read("su2_heatbath")
        or_ms, or_n = e2.profile_read("su2_overrelax")
        e2.profile(False)
        e2.close()
        d2 = diagnostics(series, 100)[0]
        out["su2_10^4_beta2.3_kp+3or"] = {
            "link_steps_per_s": world * 40000 * 4 * 500 / secs, "ms_per_sweep": 1e3 * secs / 500,
            "plaquette_mean": float(series.mean()), "plaquette_ess_per_s": world * d2.effective_sample_size / secs,
            "heatbath_us_per_launch": 1e3 * hb_ms / max(1, hb_n),
            "overrelax_us_per_launch": 1e3 * or_ms / max(1, or_n),
            "note": "200 + 500 sweeps from a cold start, plaquette every sweep into a device series "
                    "(ym_su2_measured_sweeps: one captured graph per measurement, one read-back at "
                    "the end); per-launch times from 20 further sweeps under CUDA events (1.28 MB "
                    "lattice, L2-resident: absolute rates, not an HBM fraction)"}
        # SU(3) 64 x 4^4 beta=6.0 FP64, generator uniform in 1..8, half width 0.3
        seeds = [derive_su3_chain_seed(MASTER_SEED, rank * 64 + i) for i in range(64)]
        e1 = ymgpu.Ensemble([[4, 4, 4, 4]] * 64, BETA, seeds, device=local)
        e1.metropolis_sweeps(1.0, 1000, "uniform")
        e1.synchronize()
        t = time.perf_counter()
        s1 = e1.measured_sweeps(ANGLE, 1000, 1, "uniform")
        secs = time.perf_counter() - t
        path = e1.sweep_path
        layout = e1.sweep_layout
        e1.close()
        d1 = [diagnostics(s1[:, c], 100)[0] for c in range(64)]
        m1 = s1.mean(0)
        out["su3_64x4^4_fp64_uniform_0.3"] = {
            "link_updates_per_s": world * 64 * 1024 * 1000 / secs, "us_per_sweep": 1e6 * secs / 1000,
            "plaquette_ess_per_s": world * sum(d.effective_sample_size for d in d1) / secs,
            "tau_int": float(np.mean([d.integrated_autocorrelation_time for d in d1])),
            "plaquette_mean": float(m1.mean()), "plaquette_error": float(m1.std(ddof=1) / 8.0),
            "sweep_path": path, "sweep_layout": layout,
            "note": "1000 measured sweeps (plaquette each) after 1000 at half width 1.0; one handle, "
                    "graph-replayed or chain-resident, and the sub-sweep layout, as the handle's "
                    "tuner chose"}
        # scalar-glueball pipeline, batched uneven chains, beta=5.7
        from ymgpu.pipelines import scalar_glueball_pipeline
        t = time.perf_counter()
        r = scalar_glueball_pipeline(thermalization=64, measurements=4, sweeps_between_measurements=4,
                                     device=local)
        secs = time.perf_counter() - t
        out["glueball_pipeline_128x4^3x10+64x6^3x12+32x8^3x16"] = {
            "seconds": secs, "sweep_seconds": r.sweep_seconds, "measure_seconds": r.measure_seconds,
            "prepare_seconds": r.prepare_seconds,
            "link_updates_per_s_in_sweeps": r.link_updates / r.sweep_seconds,
            "surfaces": len(r.surfaces), "sweep_layout": r.sweep_layout, "sweep_path": r.sweep_path,
            "note": "64 thermalisation sweeps (the first 50 probe the sub-sweep layouts), "
                    "4 measurements 4 sweeps apart; each measurement stout 0/5/10 levels (rho 0.1, "
                    "smeared incrementally: 10 levels in all), stride-2 blocking of the 6^3 and 8^3 "
                    "groups, A1++ operators; correlators, jackknife and covariance on the host; "
                    "prepare_seconds: the measurement graph built and uploaded once before the "
                    "first measurement"}
        # the reference's phase-3F production campaign (16 x 4^3x10, beta 5.7) with
        # its correlated fits, and the published-baseline acceptance harnesses
        from ymgpu import benchmarks as B
        from ymgpu import production as P
        campaigns = {}
        P.run_campaign(P.CAMPAIGNS["phase3f"], device=local)   # untimed: first-use setup
        for name, c in P.CAMPAIGNS.items():
            t = time.perf_counter()
            ps = P.run_campaign(c, device=local)
            secs = time.perf_counter() - t
            total = c.expected_proposals_per_chain * c.chain_count
            campaigns[name] = {
                "chains": f"{c.chain_count} x {'x'.join(map(str, c.extents))}", "seconds": secs,
                "proposals": total, "proposals_per_s": total / secs,
                "surface_outcomes": [f"{r.outcome.transformation}/{r.outcome.operator}: "
                                     + ("fit m=%.4f+-%.4f" % (r.outcome.fit.fitted_mass,
                                                              r.outcome.fit.mass_standard_error)
                                        if r.outcome.fit else r.outcome.error_code)
                                     for r in ps.surfaces],
                "scalar_pipeline_validated": ps.scalar_pipeline_validated,
                "matches_reference_observed_receipt": (P.observed_receipt_matches(ps, c)
                                                       if c.observed_outcomes else "no receipt recorded")}
        campaigns["note"] = ("each campaign: 64 + 4 sweeps per chain on the device, stout 0/1/2 "
                             "(and stride-2 blocking for 3H/3I), A1++ operators; correlators, "
                             "jackknife and the correlated fits on the host; seconds include all of it")
        out["glueball_production_campaigns"] = campaigns
        harness = {}
        for name, fn, gate in (("su2_10^4_phase2b", B.run_su2_benchmark, "phase2_graduation_gate_satisfied"),
                               ("su3_4^4_phase2c2_v1", B.run_su3_benchmark, "published_su3_baseline_reproduced"),
                               ("su3_4^4_confirmation_v2", B.run_su3_confirmation,
                                "published_su3_baseline_reproduced")):
            t = time.perf_counter()
            s = fn(device=local)
            harness[name] = {"seconds": time.perf_counter() - t, "pooled_mean": s.pooled_mean,
                             "pooled_standard_error": s.pooled_standard_error,
                             "source_envelope_reproduced": s.source_envelope_reproduced,
                             "diagnostics_trustworthy": s.diagnostics_trustworthy, gate: getattr(s, gate)}
        out["published_baseline_harnesses"] = harness
        return out

    configs_extra = other_configs()

    # end to end through the C ABI with host buffers: every step uploads a
    # lattice from pinned host memory in the reference layout, sweeps it,
    # measures its plaquette and downloads it.  E2E_LATTICES independent
    # lattices (one handle, one host buffer and one host thread each, the
    # ctypes calls releasing the interpreter lock) take turns, so while one
    # lattice uploads another downloads on the full-duplex host link and a
    # third sweeps; each thread's steps depend on its own previous download.
    # Also the same steps on one lattice alone (every transfer serialised).
    import threading
    e2e_steps = max(2 * E2E_LATTICES, min(args.steps, 10 * E2E_LATTICES)) // E2E_LATTICES * E2E_LATTICES
    lattices = [ens] + [ens.like() for _ in range(E2E_LATTICES - 1)]
    for i, h in enumerate(lattices[1:], 1):
        ens.copy_to(h)
        h.sweep_index = ens.sweep_index + 1000 * i
    hosts = []
    for h in lattices:
        h.measured_sweeps(ANGLE, 1, 1, "ordered")   # builds the handle's step graph before timing
        buf = torch.empty(links * 18, dtype=torch.float64, pin_memory=True)
        hosts.append(buf.numpy().view(np.complex128).reshape(links, 3, 3))
        h.download(0, hosts[-1])

    def e2e_step(h, host_np):
        h.upload(0, host_np)
        h.measured_sweeps(ANGLE, 1, 1, "ordered")   # one sweep, its plaquette read back
        h.download(0, host_np)

    def e2e_worker(i, n, gate):
        gate.wait()
        for _ in range(n):
            e2e_step(lattices[i], hosts[i])

    gate = threading.Barrier(E2E_LATTICES + 1)
    workers = [threading.Thread(target=e2e_worker, args=(i, e2e_steps // E2E_LATTICES, gate))
               for i in range(E2E_LATTICES)]
    for w in workers:
        w.start()
    barrier()
    gate.wait()
    t0 = time.perf_counter()
    for w in workers:
        w.join()
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0)
    barrier()
    t2 = time.perf_counter()
    for _ in range(e2e_steps // E2E_LATTICES):
        e2e_step(ens, hosts[0])
    t3 = time.perf_counter()
    e2e_one_s = max_over_ranks(t3 - t2)
    e2e = {"value": world * links * e2e_steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": links * LINK_BYTES,
           "d2h_bytes_per_step": links * LINK_BYTES + 8,
           "steps": e2e_steps,
           "path": "ym_ensemble_upload -> ym_su3_measured_sweeps (one sweep and its plaquette) "
                   f"-> ym_ensemble_download (pinned host lattice in the reference layout), {E2E_LATTICES} "
                   f"independent lattices on {E2E_LATTICES} host threads taking turns",
           "one_lattice": {"value": world * links * (e2e_steps // E2E_LATTICES) / e2e_one_s, "unit": UNIT,
                           "steps": e2e_steps // E2E_LATTICES,
                           "note": "the same steps on one lattice: upload, sweep, plaquette and "
                                   "download strictly in turn"}}
    for h in lattices[1:]:
        h.close()
    ens.close()

    if rank == 0:
        cpu = None if (args.no_cpu_baseline or world > 1) else cpu_baseline()
        line = {
            "metric": METRIC, "value": leg["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "SU(3) 32^4 beta=6.0 plain FP64 Metropolis, 8 ordered hits/link, "
                                   f"half width 0.3, Haar hot start + {args.thermalization} untimed "
                                   "wide-angle sweeps",
                       "lattice": "32^4", "global_batch": world, "parallelism": f"replicas x{world}",
                       "l2": "inputs 604 MB > 126 MB L2 (no flush)",
                       "step": "1 checkerboard sweep + average plaquette (run_chain cadence through "
                               "ym_su3_measured_sweeps: one captured graph per step, plaquettes kept in a "
                               "device series and read back once)"},
            "plaquette_mean": float(np.mean(plaq)),
            "acceptance": leg["acceptance"],
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            # measured steps: 8 sub-sweeps (3 measuring), sweep counter, reduction, series store;
            # per-launch steps: 8 sub-sweeps, sweep counter, plaquette, reduction
            "gpu_launches": int((args.steps - leg["roofline"]["per_launch_steps"]) * 11
                                + leg["roofline"]["per_launch_steps"] * 11),
            "clocks": leg["clocks"],
            "clocks_leg": dict(leg["clocks_leg"] or {}, note="every sample of the FP64 leg: "
                               "warm-up, timed steps and the sampler's start and stop"),
            "fp32_two_row": {
                "value": f32["value"], "unit": UNIT, "dtype": "f32 links, f64 dS/accept/plaquette",
                "ms_per_step": f32["ms"] / args.steps,
                "step": "1 checkerboard sweep + FP64 reunitarisation + average plaquette",
                "plaquette_mean": float(np.mean(f32["plaq"])), "acceptance": f32["acceptance"],
                "roofline": f32["roofline"]},
            "fp64_fast": {
                "value": fleg["value"], "unit": UNIT, "ms_per_step": fleg["ms"] / args.steps,
                "dtype": "f64 (fused multiply-adds, Horner rotations)",
                "step": "1 checkerboard sweep (fast form) + average plaquette",
                "plaquette_mean": float(np.mean(fleg["plaq"])), "acceptance": fleg["acceptance"],
                "roofline": dict(fleg["roofline"], kernel="tiled_fast::k_su3_metropolis_ring "
                                                          "(ordered hits; one sub-sweep)"),
                "error_vs_exact": fast_err},
            "learned": {
                "value": lrn["value"], "unit": UNIT, "ms_per_step": lrn["ms"] / args.steps,
                "dtype": "f32 links, bf16 network (fp32 accumulate), f64 dS/accept/plaquette",
                "step": "1 learned checkerboard sweep + FP64 reunitarisation + average plaquette",
                "plaquette_mean": float(np.mean(lrn["plaq"])), "acceptance": lrn["acceptance"],
                "roofline": dict(lrn["roofline"], kernel="k_lp_sweep (staple, features, tcgen05 "
                                                         "network, 8 hits; one sub-sweep)"),
                "training": {"configurations": args.train_steps, "seconds": train_s,
                             "geometry": f"{ESS_CHAINS} x 16^4", "lr": TRAIN_LR,
                             "objective_first": float(np.mean(train_hist[:20])),
                             "objective_last": float(np.mean(train_hist[-20:])),
                             "mean_half_width": float(np.mean(s_half)),
                             "mean_generator_probabilities": [float(v) for v in p_gen.mean(0)]}},
            "other_configs": configs_extra,
            "stout_32x4_fp64": stout,
            "observables_32x4_fp64": observables,
            "loop_cadence_fp32_vs_fp64": loop_runs,
            "ess": {
                "geometry": f"{ESS_CHAINS} chains x 16^4 (total volume of 32^4), beta=6.0, "
                            f"{n} measured sweeps per sampler from one equilibrated state",
                "estimator": "reference diagnostics (initial positive window), per chain, summed",
                "plain_f64_ordered_0.3": ess_f64, "plain_f32_uniform_0.3": ess_f32,
                "plain_f32_uniform_1.0": ess_f32w, "learned_f32": ess_lrn,
                "plain_f32_uniform_at_learned_scale": ess_f32c,
                "control_note": "plain_f32_uniform_1.0 is plain Metropolis at the widest half "
                                "width the reference admits; plain_f32_uniform_at_learned_scale "
                                "is plain Metropolis with uniform generators at the constant "
                                "half width the trained network settles at (the matched "
                                "control: same scale, no per-link network)",
                "learned_vs_constant_scale": ess_lrn["plaquette_ess_per_s"] /
                                             ess_f32c["plaquette_ess_per_s"],
                "tau_learned_vs_constant_scale": ess_lrn["tau_int"] / ess_f32c["tau_int"],
                "plaquette_sigma_learned_vs_constant_scale": float(sig(ess_lrn, ess_f32c)),
                "learned_vs_plain_f32_at_1.0": ess_lrn["plaquette_ess_per_s"] /
                                               ess_f32w["plaquette_ess_per_s"],
                "learned_vs_plain_f64": ess_lrn["plaquette_ess_per_s"] / ess_f64["plaquette_ess_per_s"],
                "learned_vs_plain_f32": ess_lrn["plaquette_ess_per_s"] / ess_f32["plaquette_ess_per_s"],
                "learned_vs_plain_f64_with_training": (
                    (ess_lrn["plaquette_ess_per_s"] * ess_lrn["seconds"]) /
                    (ess_lrn["seconds"] + train_s)) / ess_f64["plaquette_ess_per_s"],
                "plaquette_sigma_learned_vs_f64": float(sig(ess_lrn, ess_f64)),
                "plaquette_sigma_f32_vs_f64": float(sig(ess_f32, ess_f64))},
        }
        rep.emit(line)
    rep.close()


if __name__ == "__main__":
    main()
