"""Query sharding over GPUs (one process per GPU, torch.distributed).

Queries are independent, so a batch splits into contiguous slices, one per
rank; every rank answers its slice on its own replica of the cloud (built from
the same points, or restored from a checkpoint) and the slices' results are
gathered.  The search itself has no collective; the gather is two all_gather
calls (sizes, then the padded results).  With the NCCL backend the tensors are
CUDA tensors, with gloo host tensors.

The reference has no counterpart: it answers queries on OpenMP threads of one
host (neighbor_benchmarks.hpp:518-567).
"""
from __future__ import annotations


def shard_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """[begin, end) of rank's slice of n queries: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(int(n), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def _gather_padded(t, group=None):
    """all_gather of tensors whose first dimension differs by rank; returns the list, unpadded."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes) if sizes else 0
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[: t.shape[0]] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return [p[:s] for p, s in zip(parts, sizes)]


def gather_csr(offsets, indices, group=None):
    """The CSR results of every rank's slice (offsets from 0, length m + 1; indices), in rank order, as one
    CSR result on every rank: (offsets int64, indices)."""
    import torch

    counts = offsets[1:] - offsets[:-1]
    all_counts = _gather_padded(counts.to(torch.int64), group)
    all_idx = _gather_padded(indices[: int(offsets[-1].item())] if offsets.numel() > 1 else indices[:0], group)
    cnt = torch.cat(all_counts)
    out = torch.zeros(cnt.shape[0] + 1, dtype=torch.int64, device=cnt.device)
    torch.cumsum(cnt, 0, out=out[1:])
    return out, torch.cat(all_idx)


def gather_rows(*tensors, group=None):
    """Row-wise results of every rank's slice (kNN indices, squared distances, counts), concatenated in rank
    order on every rank."""
    import torch

    return tuple(torch.cat(_gather_padded(t, group)) for t in tensors)
