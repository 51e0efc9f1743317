"""The N > 1 path of bench.py on the CPU: one independent replica per rank
(the dense solve does not shard), whole-job figures from a max-over-ranks
step time.  Two gloo ranks stand in for two GPUs."""
import datetime
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, ms_by_rank, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench
        step = bench.replicas_aggregate(ms_by_rank[rank], 1000.0, ws, torch.device("cpu"))
        e2e = bench.replicas_aggregate(ms_by_rank[rank] + 1.0, 1000.0, ws, torch.device("cpu"))
        dist.barrier()
        out.put((rank, step, e2e))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_rank_and_sum_the_units():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ms_by_rank = [10.0, 12.5]
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ms_by_rank, out)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(out.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    for rank, (ms, value), (e2e_ms, e2e_value) in got:
        assert ms == 12.5 and value == pytest.approx(2 * 1000.0 / 12.5e-3)
        assert e2e_ms == 13.5 and e2e_value == pytest.approx(2 * 1000.0 / 13.5e-3)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replicas_aggregate(4.0, 500.0, 1, "cpu") == (4.0, pytest.approx(500.0 / 4e-3))


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm's other ranks exit 0 without work."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def _sweep_worker(rank, ws, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench
        ks = [16.0 + i / 30.0 for i in range(7)]
        mine = bench.shard_wavenumbers(ks, rank, ws)
        # per-k results a rank computes for its own wavenumbers
        local = {"k": list(mine), "twice": [2.0 * k for k in mine]}
        merged = bench.sweep_gather(local, ks, rank, ws)
        out.put((rank, mine, merged))
    finally:
        dist.destroy_process_group()


def test_sweep_shards_wavenumbers_and_gathers_in_order():
    """The sweep workload on N ranks: rank r takes k_r, k_(r+N), ..., every k
    exactly once, and the per-k results come back in the sweep's k order."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ws = 3
    procs = [ctx.Process(target=_sweep_worker, args=(r, ws, port, out)) for r in range(ws)]
    for p in procs:
        p.start()
    try:
        got = sorted((out.get(timeout=120) for _ in procs), key=lambda t: t[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0] * ws
    ks = [16.0 + i / 30.0 for i in range(7)]
    shares = [mine for _, mine, _ in got]
    assert sorted(k for sh in shares for k in sh) == ks and shares[0] == [ks[0], ks[3], ks[6]]
    for _, _, merged in got:
        assert merged["k"] == ks and merged["twice"] == [2.0 * k for k in ks]


def test_sweep_gather_on_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench
    ks = [1.0, 2.0, 3.0]
    assert bench.shard_wavenumbers(ks, 0, 1) == ks
    assert bench.sweep_gather({"x": [5, 6, 7]}, ks, 0, 1) == {"x": [5, 6, 7]}
