"""The multi-GPU path of bench.py on CPU: world_size-2 gloo ranks.

B64 splits whole systems over the ranks (no collective in the solve); the
ranks then agree on the timing through a max all-reduce. Both steps run here
with the gloo backend on 127.0.0.1, as they run under torchrun with NCCL."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, rows, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = bench.shard_systems(rows, world, rank)
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        t = torch.tensor([float(10 + rank)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out.put((rank, parts, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_b64_sharding_over_two_gloo_ranks():
    import multiprocessing as mp
    import gpusolver_b200 as gs
    import bench
    u = gs.uniform_rhs(bench.B64_SYSTEMS, bench.B64_SEED)
    sides = [16 + min(80, int((v + 1.0) / 2.0 * 81)) for v in u]
    rows = [m ** 3 for m in sides]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, rows, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, parts, tmax in results:
        assert tmax == 11.0  # max over ranks
        flat = sorted(i for part in parts for i in part)
        assert flat == list(range(len(rows)))  # every system on exactly one rank
        loads = [sum(rows[i] for i in part) for part in parts]
        assert abs(loads[0] - loads[1]) <= max(rows)  # greedy balance bound
    assert results[0][1] == results[1][1]  # both ranks computed the same split
