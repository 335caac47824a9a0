"""Query sharding over GPUs (one process per GPU, torch.distributed).

Queries are independent, so a batch splits into contiguous slices, one per
rank; every rank answers its slice on its own replica of the cloud (built from
the same points, or restored from a checkpoint) and the slices' results are
gathered.  The search itself has no collective; the gather is two all_gather
calls (sizes, then the padded results).  With the NCCL backend the tensors are
CUDA tensors, with gloo host tensors.  A replica either builds from the same
points on every rank or is restored from the checkpoint one rank built and
broadcast (broadcast_checkpoint).

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


def broadcast_checkpoint(ck, src: int = 0, group=None):
    """A built cloud's checkpoint (LinearOctree.checkpoint(): a dict of host arrays) from rank `src` (its
    rank in the default group) to every rank, so that one rank sorts and builds and the others restore
    the same tree with LinearOctree.from_checkpoint instead of building it again.  Ranks other than src
    pass None.  Returns the checkpoint on every rank, each value a numpy array (0-d for scalars).

    One broadcast carries the names, dtypes and shapes, then one broadcast per non-empty array carries its
    raw bytes, so every dtype crosses unchanged.  With the NCCL backend the bytes go through this rank's
    current CUDA device (over NVLink between the GPUs), with gloo they stay on the host.  Every rank makes
    the same calls in the same order."""
    import numpy as np
    import torch
    import torch.distributed as dist

    is_src = dist.get_rank() == src
    if is_src:
        if ck is None:
            raise ValueError("the source rank must pass the checkpoint")
        arrays = {}
        for k, v in ck.items():
            a = np.asarray(v)
            arrays[str(k)] = a if a.flags.c_contiguous else np.ascontiguousarray(a)  # keeps 0-d scalars 0-d
        meta = [(k, a.dtype.str, tuple(a.shape)) for k, a in arrays.items()]
    else:
        arrays, meta = {}, None
    box = [meta]
    dist.broadcast_object_list(box, src=src, group=group)
    meta = box[0]
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else None
    out = {}
    for name, dt, shape in meta:
        dtype = np.dtype(dt)
        nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
        if nbytes == 0:
            out[name] = np.zeros(shape, dtype)
            continue
        if is_src:
            buf = torch.from_numpy(arrays[name].reshape(-1).view(np.uint8))
        else:
            buf = torch.empty(nbytes, dtype=torch.uint8)
        moved = buf.to(dev) if dev is not None else buf
        dist.broadcast(moved, src=src, group=group)
        if is_src:
            out[name] = arrays[name]
        else:
            host = moved.cpu() if dev is not None else moved
            out[name] = host.numpy().view(dtype).reshape(shape).copy()
    return out
