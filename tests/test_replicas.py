"""The multi-GPU path on the CPU: two ranks over gloo exercise the replica
plumbing bench.py uses (barrier, slowest-rank timing, per-rank seeds,
rank-0 output), a rank that dies before a collective ends the other's wait
with an error instead of a hang, and the reference arm under torchrun
prints one line from rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path, fail_rank, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "yang-mills_b200"))
    try:
        from ymgpu.replicas import Replicas
        rep = Replicas(backend="gloo", timeout_s=5.0)
        if rank == fail_rank:
            q.put((rank, "left"))
            q.close()
            q.join_thread()        # the message is out before the process dies
            os._exit(3)            # dies without joining the next collective
        rep.barrier()
        m = rep.max_over_ranks(1.5 + rank)
        s = rep.sum_over_ranks(1.0 + rank)
        seed = rep.chain_seed(0x2C02198105010002)
        with open(out_path, "a") as fh:
            rep.emit({"rank": rank, "max": m, "sum": s, "value": rep.weak_value(100.0, m)}, fh)
        rep.close()
        q.put((rank, {"max": m, "sum": s, "seed": seed}))
    except Exception as e:     # the surviving rank of a failure test lands here
        q.put((rank, f"error: {type(e).__name__}"))


def _run(world, fail_rank, tmp_path):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    out = os.path.join(tmp_path, "lines.jsonl")
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out, fail_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=90)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung"
    res = {}
    while not q.empty():
        r, v = q.get()
        res[r] = v
    return res, out


def test_two_gloo_ranks_reduce_and_print_once(tmp_path):
    from ymgpu.su3_ensemble import derive_su3_chain_seed
    res, out = _run(2, -1, tmp_path)
    assert res[0]["max"] == res[1]["max"] == 2.5
    assert res[0]["sum"] == res[1]["sum"] == 3.0
    assert res[0]["seed"] == derive_su3_chain_seed(0x2C02198105010002, 0)
    assert res[1]["seed"] == derive_su3_chain_seed(0x2C02198105010002, 1)
    lines = open(out).read().splitlines()
    assert len(lines) == 1 and json.loads(lines[0]) == {"rank": 0, "max": 2.5, "sum": 3.0,
                                                        "value": 2 * 100.0 / 2.5}


def test_a_rank_that_dies_ends_the_other_wait_with_an_error(tmp_path):
    res, _ = _run(2, 1, tmp_path)
    assert res[1] == "left"
    assert isinstance(res[0], str) and res[0].startswith("error"), res[0]


def test_reference_arm_under_torchrun_prints_from_rank_zero_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
