"""DB sharding across GPUs and the result exchange between shards.

The reference spreads the share DB over the GPUs of a party round-robin: global
entry g lives on device g % n at local index g // n (iris-mpc-gpu/src/server/
actor.rs:852-853 for reauth targets, 2648-2649 for deletions, 2693-2694 for
updates, 3681 for insertions).  Every device scans its own shard for the whole
query batch, with no data exchanged during the scan; afterwards the per-device
results are merged: the first match of a query is the smallest global index
over all devices (get_merged_results, actor.rs:3174-3196), and the match lists
are the union of the devices' lists mapped to global indices.

Here one process drives one GPU; the merge runs as one all_gather over
torch.distributed (NCCL between GPUs, gloo on CPU), after which every rank
holds the merged results.
"""
from __future__ import annotations

import numpy as np

NON_MATCH_ID = 0xFFFFFFFF


def global_id(local, rank: int, world: int):
    """Global entry index of local index `local` on shard `rank`."""
    return np.asarray(local, np.int64) * world + rank


def shard_of(gid, world: int):
    """(rank, local index) of global entry `gid`."""
    g = np.asarray(gid, np.int64)
    return g % world, g // world


def shard_len(total: int, rank: int, world: int) -> int:
    """Entries of a `total`-entry DB that live on shard `rank`."""
    return max(0, (total - rank + world - 1) // world)


def shard_entries(total: int, rank: int, world: int) -> np.ndarray:
    """Global indices held by shard `rank`, in local order."""
    return np.arange(rank, total, world, dtype=np.int64)


def append_target(total: int, world: int):
    """(rank, local index) where the next appended entry (global index
    `total`) is written."""
    return int(total % world), int(total // world)


def merge_final_results(per_rank_final) -> np.ndarray:
    """get_merged_results: per_rank_final[r][q] is the first local match of
    query q on shard r (NON_MATCH_ID if none); returns the smallest global
    index per query (NON_MATCH_ID if no shard matched)."""
    world = len(per_rank_final)
    out = np.full(len(per_rank_final[0]), NON_MATCH_ID, np.int64)
    for r, f in enumerate(per_rank_final):
        f = np.asarray(f, np.int64)
        g = np.where(f != NON_MATCH_ID, f * world + r, NON_MATCH_ID)
        out = np.minimum(out, g)
    return out.astype(np.uint32)


def merge_match_lists(per_rank_counts, per_rank_ids, cap: int | None = None):
    """Union of the shards' match lists, as sorted global indices per query.
    per_rank_ids[r][q] holds the first min(count, width) local matches of
    query q on shard r (width = the list's length).  Returns (total counts,
    [sorted global ids per query]).

    Each list keeps at most min(cap, width) ids (width alone when cap is
    None): a shard's ids beyond its width are unknown, so only the smallest
    `width` merged ids are certain to be the smallest global matches (every
    one of them is among its own shard's smallest `width`).  A query whose
    total count exceeds its list's length was truncated."""
    world = len(per_rank_counts)
    nq = len(per_rank_counts[0])
    counts = np.zeros(nq, np.int64)
    lists = []
    for q in range(nq):
        ids = []
        width = min(len(per_rank_ids[r][q]) for r in range(world))
        for r in range(world):
            n = int(per_rank_counts[r][q])
            counts[q] += n
            local = np.asarray(per_rank_ids[r][q][: min(n, len(per_rank_ids[r][q]))], np.int64)
            ids.append(local * world + r)
        merged = np.sort(np.concatenate(ids)) if ids else np.zeros(0, np.int64)
        keep = width if cap is None else min(cap, width)
        lists.append(merged[:keep])
    return counts, lists


def exchange_results(final, counts, ids, group=None, device=None):
    """All-gathers every rank's (final [nq], counts [nq], ids [nq][w]) u32
    results and returns the merged (final, counts, lists) on every rank.  One
    collective for the three arrays; NCCL needs `device` (a cuda device) and
    gloo runs on CPU tensors."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    final = np.asarray(final, np.int64)
    counts = np.asarray(counts, np.int64)
    ids = np.asarray(ids, np.int64)
    nq, w = ids.shape
    packed = np.concatenate([final[:, None], counts[:, None], ids], axis=1)  # [nq][2 + w]
    t = torch.from_numpy(packed)
    if device is not None:
        t = t.to(device)
    bufs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(bufs, t, group=group)
    parts = [b.cpu().numpy() for b in bufs]
    merged_final = merge_final_results([p[:, 0] for p in parts])
    mc, lists = merge_match_lists([p[:, 1] for p in parts], [p[:, 2:] for p in parts])
    return merged_final, mc, lists
