"""The multi-GPU replica path on CPU: two gloo ranks (127.0.0.1), distinct
seeds, MAX-over-ranks timing and the whole-job throughput -- the same code
bench.py uses with NCCL, no GPU needed."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from fpga_mps_simulator_b200.replicas import Replicas
    r = Replicas(backend="gloo", timeout_s=60)
    seconds = 1.0 + rank          # rank 1 is the slow one
    r.barrier()
    q.put((rank, r.seed(2024), r.max(seconds), r.throughput(990, seconds)))
    r.close()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2024, 2025]
    assert all(o[2] == 2.0 for o in out)
    assert all(abs(o[3] - 2 * 990 / 2.0) < 1e-12 for o in out)


def test_single_process_needs_no_group():
    from fpga_mps_simulator_b200.replicas import Replicas
    r = Replicas(backend="gloo")
    assert (r.rank, r.world) == (0, 1)
    assert r.max(3.5) == 3.5
    assert r.throughput(10, 2.0) == 5.0
    r.close()
