"""Root-partitioned counting across GPUs: one process per GPU.

FFS subtrees under different root candidates are independent, so each rank
counts the embeddings whose root lies in its degree-balanced part of every
query's root window (gfsm_batch_count_part) against its own copy of the data
graph, and one 8-byte count per query is summed over the ranks with an
all-reduce.  No other data crosses between GPUs.  The reference runs its FFS
on one GPU; this has no counterpart there.
"""
import numpy as np


def count_partitioned(ctx, plans, data, group=None):
    """Whole-job counts of `plans` on `data`: this rank's part of every root
    window, summed over the process group.  Returns (counts, this rank's
    stats).  The tensor for the all-reduce lives on the rank's CUDA device
    under NCCL and on the CPU under gloo."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    counts, st = ctx.batch_count_part(plans, data, rank, world)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(counts.astype(np.int64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy().astype(np.uint64), st
