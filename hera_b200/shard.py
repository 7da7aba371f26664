"""Multi-GPU work split: one process per GPU, each with its own replica of
the index, read chunks dealt round robin, no collective on the data path.

hera's per-chunk results are consumed in input order by its host tail
(add_class order fixes the EM's class order), so the only exchange is an
ordered merge of per-chunk results on one rank -- the records, or only the
per-chunk class tables when the ranks build those on their devices -- plus
the max-over-ranks of the device timing.  Both are small host-side steps
over torch.distributed (gloo on CPU, nccl on GPUs).
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


def merge_class_tables(tables: List[Any]):
    """Per-chunk class tables (each built from one chunk's records alone,
    given in chunk order) -> the table hera's add_class builds over all
    chunks in order (src/hash_align.c:1564-1602).  A class first seen in
    chunk c is numbered after every class of earlier chunks and, among
    chunk c's new classes, in chunk c's own first-insertion order, keeping
    chunk c's transcript list; counts, REF_INF->count, PAIRED and the
    fragment sum add up.  Tables need ids, counts, ns, ref_off, ref,
    tx_count, paired and mean_frag (hera_b200.api.ClassTable has them)."""
    import numpy as np
    from .api import ClassTable
    if not tables:
        raise ValueError("no class tables")
    index = {}
    ids, counts, ns, lists = [], [], [], []
    tx = np.zeros_like(np.asarray(tables[0].tx_count, dtype=np.uint64))
    paired, frag = 0, 0.0
    for t in tables:
        ref = np.asarray(t.ref)
        for k, cid in enumerate(np.asarray(t.ids).tolist()):
            j = index.get(cid)
            if j is None:
                index[cid] = len(ids)
                ids.append(cid)
                counts.append(float(t.counts[k]))
                ns.append(int(t.ns[k]))
                o = int(t.ref_off[k])
                lists.append(ref[o:o + int(t.ns[k])])
            else:
                counts[j] += float(t.counts[k])
        tx += np.asarray(t.tx_count, dtype=np.uint64)
        paired = (paired + int(t.paired)) & 0xFFFFFFFF   # PAIRED is an unsigned int
        frag += float(t.mean_frag)
    off = np.zeros(len(ns), np.uint64)
    if ns:
        off[1:] = np.cumsum(np.asarray(ns[:-1], np.uint64))
    ref = np.concatenate(lists).astype(np.uint32) if lists else np.zeros(0, np.uint32)
    return ClassTable(np.asarray(ids, np.uint32), np.asarray(counts, np.float64), np.asarray(ns, np.uint32),
                      off, ref, (tx & 0xFFFFFFFF).astype(np.uint32), paired, frag)
