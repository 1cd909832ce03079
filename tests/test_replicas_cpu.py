"""Host logic of the multi-GPU runs (one process per GPU, independent work per rank),
exercised with two gloo ranks on the CPU: max-over-ranks timing, whole-job throughput,
the cell-count partition of independent problems, gathering per-rank results, and the
partition -> per-rank solve -> gather flow of the batched shock tubes on tiny problems
(solved on each rank by the CPU restatement, which stands in for the GPU batch here)."""
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


def _tubes():
    from subfv_b200 import shocktube
    return shocktube.sample(6, seed=3, n_min=8, n_max=24)


def _solve_tubes(indices):
    """Each problem to its end time on this rank (first-order multi_point, CFL 0.4)."""
    import time
    import numpy as np
    from oracle.oracle import OracleMesh
    from subfv_b200 import shocktube
    from subfv_b200.ns import NsConfig
    tubes = _tubes()
    out, units, t0 = [], 0, time.perf_counter()
    for i in indices:
        raw = shocktube.raw_mesh(tubes[i])
        o = OracleMesh(raw)

        class _M:  # what initial_state reads of a mesh
            n_elems = o.n_elems

            def geometry(self, name, o=o):
                return o.geom(name)
        sol = np.ascontiguousarray(shocktube.initial_state(_M(), tubes[i]))
        cfg = NsConfig(scheme=1, second_order=False, method=4, bc_style=2, boundary_2d=True, cfl=0.4,
                       tmax=tubes[i].t_end)
        st, it, t, _, _, _ = o.ns_run(cfg.oracle_dict(), sol, 10 ** 6)
        out.append((st, it, sol.tobytes()))
        units += o.n_elems * it
    return out, units, time.perf_counter() - t0


def _worker_partitioned(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from subfv_b200 import replicas
        sizes = [t.n_cells for t in _tubes()]
        res, rate, sec = replicas.run_partitioned(sizes, _solve_tubes)
        q.put((rank, res, rate, sec))
    finally:
        dist.destroy_process_group()


def test_partitioned_shock_tubes_two_gloo_ranks():
    world, port = 2, 30617 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker_partitioned, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=120) for _ in ps), key=lambda x: x[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    alone, _, _ = _solve_tubes(list(range(len(_tubes()))))
    for rank, got, rate, sec in res:
        assert got == alone  # every problem, in problem order, as solved on one rank
        assert rate > 0 and sec > 0
    assert res[0][2] == res[1][2]  # the same whole-job figure on every rank
