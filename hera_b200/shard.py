"""Multi-GPU work split: one process per GPU, each with its own replica of
the index, read chunks dealt round robin, no collective on the data path.

hera's per-chunk results are consumed in input order by its host tail
(add_class order fixes the EM's class order), so the only exchange is an
ordered merge of per-chunk results on one rank, plus the max-over-ranks of
the device timing.  Both are small host-side steps over torch.distributed
(gloo on CPU, nccl on GPUs).
"""
from __future__ import annotations

from typing import Any, Dict, List


def chunk_ids(n_chunks: int, rank: int, world: int) -> List[int]:
    """Chunks this rank aligns: rank, rank + world, rank + 2*world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(range(rank, n_chunks, world))


def merge_in_order(parts: List[Dict[int, Any]], n_chunks: int) -> List[Any]:
    """Per-rank {chunk id: result} maps -> results in chunk order; every
    chunk must appear exactly once."""
    out: List[Any] = [None] * n_chunks
    seen = [False] * n_chunks
    for part in parts:
        for cid, res in part.items():
            if not 0 <= cid < n_chunks or seen[cid]:
                raise ValueError(f"chunk {cid} missing or duplicated")
            seen[cid] = True
            out[cid] = res
    if not all(seen):
        raise ValueError(f"chunks {[i for i, s in enumerate(seen) if not s]} missing")
    return out


def gather_in_order(local: Dict[int, Any], n_chunks: int, dst: int = 0):
    """Gather every rank's {chunk id: result} on `dst` and return the merged
    chunk-ordered list there (None elsewhere)."""
    import torch.distributed as dist
    world = dist.get_world_size()
    parts = [None] * world if dist.get_rank() == dst else None
    dist.gather_object(local, parts, dst=dst)
    if dist.get_rank() != dst:
        return None
    return merge_in_order(parts, n_chunks)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (the slowest rank's time)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
