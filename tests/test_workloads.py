"""Instance mix and sharding of the batched workload (host logic; CPU)."""
import os

import pytest

from gemini_b200 import workloads as WL


def test_batched_specs_ranges_and_mix():
    specs = WL.batched_specs(64, seed=2024)
    assert len(specs) == 64
    assert all(64 <= s.lx1 <= 512 and 16 <= s.lx2 <= 128 and 16 <= s.lx3 <= 128 for s in specs)
    assert sum(s.kind == "dipole" for s in specs) == 32
    assert len({s.seed for s in specs}) == 64
    assert WL.batched_specs(64, seed=2024) == specs  # deterministic


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_partitions_and_balances(world):
    specs = WL.batched_specs(64, seed=7)
    parts = [WL.shard(specs, world, r) for r in range(world)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))  # every instance exactly once
    loads = [sum(specs[i].cells for i in p) for p in parts]
    biggest = max(s.cells for s in specs)
    assert max(loads) - min(loads) <= biggest  # LPT bound


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = WL.batched_specs(64, seed=3)
    mine = WL.shard(specs, world, rank)
    # the only cross-rank traffic of the batched form: a host gather of per-instance status
    status = torch.zeros(64, dtype=torch.int64)
    for i in mine:
        status[i] = 1 + i
    dist.all_reduce(status)
    cells = torch.tensor([float(sum(specs[i].cells for i in mine))], dtype=torch.float64)
    dist.all_reduce(cells)
    q.put((rank, status.tolist(), float(cells.item())))
    dist.destroy_process_group()


def test_shard_status_gather_two_ranks_gloo():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = WL.batched_specs(64, seed=3)
    for _, status, cells in res:
        assert status == [1 + i for i in range(64)]
        assert cells == float(sum(s.cells for s in specs))
