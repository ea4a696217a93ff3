"""The N>1 path of bench.py on CPU: world_size-2 gloo ranks run independent
replicas and aggregate max elapsed time and summed units (no data-path
collective: the layered-circuit path does not shard)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t, u = bench.aggregate(10.0 + 5.0 * rank, 930.0)
    q.put((rank, t, u, bench.dist_env()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_aggregation_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, u, env in out:
        assert t == 15.0 and u == 1860.0
        assert env[0] == 2 and env[1] == rank


def test_reference_arm_prints_a_line(tmp_path):
    """--impl reference runs the oracle restatement on the host (small instance)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--qubits", "12",
                        "--depth", "2", "--steps", "3", "--warmup", "1"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "gates/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
