"""Host logic of the multi-GPU runs (one process per GPU, independent work per rank),
exercised with two gloo ranks on the CPU: max-over-ranks timing, whole-job throughput,
the cell-count partition of independent problems, and gathering per-rank results."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from subfv_b200 import replicas
        m = replicas.max_over_ranks(1.5 + rank)
        thr, sec = replicas.aggregate_throughput(100.0 * (rank + 1), 2.0 + rank)
        cells = [5, 40, 7, 40, 1, 12, 3, 30]
        parts = replicas.partition_by_cells(cells, world)
        mine = parts[rank]
        got = replicas.gather_lists([(rank, i) for i in mine])
        q.put((rank, m, thr, sec, parts, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, 29517 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, m, thr, sec, parts, got in res:
        assert m == 2.5
        assert sec == 3.0 and thr == pytest.approx(300.0 / 3.0)
        assert parts == res[0][4]  # every rank computes the same partition
        assert sorted(i for _, i in got) == list(range(8))  # each problem on exactly one rank
        assert [r for r, _ in got] == sorted(r for r, _ in got)  # rank order


def test_partition_balances_and_is_deterministic():
    from subfv_b200.replicas import partition_by_cells
    cells = [100, 90, 80, 70, 60, 50, 40, 30, 20, 10]
    parts = partition_by_cells(cells, 3)
    loads = [sum(cells[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(cells) // 2
    assert partition_by_cells(cells, 3) == parts
    assert sorted(i for p in parts for i in p) == list(range(10))
    assert all(p == sorted(p) for p in parts)
    assert partition_by_cells(cells, 1) == [list(range(10))]
