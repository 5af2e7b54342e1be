"""Multi-GPU serving by replicas.

The encrypted IVF-PQ path shards by independent queries: every rank holds its
own context, keys and resident plaintexts and serves its own queries; nothing
is exchanged on the data path. The only collective is the end-of-run report:
the job's throughput is all ranks' queries over the slowest rank's device
time.
"""
from __future__ import annotations


def query_seed(base: int, rank: int) -> int:
    """Disjoint query streams per rank."""
    return base + 1000 * rank


def aggregate(local_ms: float, local_queries: int) -> tuple[float, int]:
    """(max over ranks of device milliseconds, sum over ranks of queries).

    Works with the nccl backend (tensors on the current CUDA device) and with
    gloo (CPU tensors); without an initialised process group it is the identity.
    """
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_ms), int(local_queries)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=dev)
    q = torch.tensor([int(local_queries)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(q, op=dist.ReduceOp.SUM)
    return float(t.item()), int(q.item())
