"""Replica aggregation across ranks (world size 2, gloo on CPU): the job time
is the slowest rank's, the query count the sum, and per-rank query streams
are disjoint."""
import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from anns_fhe_b200.replicas import aggregate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = aggregate(10.0 + 5 * rank, 100 + rank)
    finally:
        dist.destroy_process_group()


def test_aggregate_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == (15.0, 201)


def test_single_process_is_identity():
    from anns_fhe_b200.replicas import aggregate, query_seed
    assert aggregate(3.5, 7) == (3.5, 7)
    assert len({query_seed(1000, r) for r in range(8)}) == 8

