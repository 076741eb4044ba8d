"""Row sharding across GPUs: one process per GPU holds the fact rows
[rank * rows_per_rank, (rank + 1) * rows_per_rank) of every column (the
generator is counter-based, keyed by the global row) and builds its own
slice of the bitmap index; dimensions are replicated.  Every query's int64
group sums and row counts are additive over row ranges, so one all-reduce
(sum) of the per-rank tables is the whole exchange.

No counterpart in the reference, which runs on one GPU.
"""
from __future__ import annotations


def row_range(rank: int, rows_per_rank: int) -> tuple[int, int]:
    """(first global row, rows) of a rank's shard."""
    if rank < 0 or rows_per_rank <= 0:
        raise ValueError("rank >= 0 and rows_per_rank > 0")
    return rank * rows_per_rank, rows_per_rank


def combine(out, nqual, group=None) -> None:
    """Sums the per-rank group tables and row counts in place over the
    process group (NCCL for CUDA tensors, gloo for CPU tensors)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(nqual, op=dist.ReduceOp.SUM, group=group)
