"""The N > 1 path of bench.py: independent replicas, timing reduced as the max over ranks
(world size 2, gloo, CPU)."""
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

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sec = bench.max_over_ranks(1.0 + rank, world, "cpu")
    q.put((rank, sec, bench.replica_throughput(world, 1000, 10, sec)))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
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
    assert [o[1] for o in out] == [2.0, 2.0]
    assert out[0][2] == pytest.approx(2 * 1000 * 10 / 2.0)


def _ens_rank(rank, world, port, q):
    import torch.distributed as dist

    import bench
    from pyexner_b200.cases import ensemble_case
    from pyexner_b200.ensemble import partition_members

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    members, _ = ensemble_case(64, 0)
    cells = [m["shape"][0] * m["shape"][1] for m in members]
    mine = partition_members(cells, world)[rank]
    my_cells = sum(cells[k] for k in mine)
    total = bench.sum_over_ranks(my_cells, world, "cpu")
    sec = bench.max_over_ranks(0.5 + 0.25 * rank, world, "cpu")
    q.put((rank, mine, my_cells, total, sec, sum(cells)))
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_members_split_over_ranks():
    """The ensemble leg of bench.py under two ranks: every member on exactly one rank,
    the shares balanced, whole-job cells summed and the time the slowest rank's."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ens_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, c0, t0, s0, all0), (_, m1, c1, t1, s1, all1) = out
    assert sorted(m0 + m1) == list(range(64)) and not set(m0) & set(m1)
    assert t0 == t1 == c0 + c1 == all0 == all1
    assert s0 == s1 == 0.75
    assert abs(c0 - c1) <= 0.05 * (c0 + c1)


def test_partition_members_is_deterministic_and_balanced():
    from pyexner_b200.ensemble import partition_members

    cells = [5, 9, 1, 7, 7, 3, 2, 8]
    for world in (1, 2, 3, 4, 8, 10):
        parts = partition_members(cells, world)
        assert len(parts) == world
        assert sorted(k for p in parts for k in p) == list(range(len(cells)))
        assert parts == partition_members(cells, world)
        loads = [sum(cells[k] for k in p) for p in parts]
        if world <= len(cells):
            assert max(loads) - min(loads) <= max(cells)
