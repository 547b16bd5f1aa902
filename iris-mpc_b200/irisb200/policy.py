"""OR-policy bitmaps for the two-eye merge.

The reference decides, per (query, DB entry), whether a match needs both eyes
(AND, the default) or either eye (OR): the OR rule applies to DB entries listed
per query, plus, unless a request opts out, the most recent records of the DB
(the lookback window).  prepare_or_policy_bitmap and generate_luc_records
(iris-mpc-gpu/src/server/actor.rs:3601-3660) build that bitmap on the host; it
is then passed to the merge (irs_dc_join_db_matches, mergeDbResultsWithOr-
PolicyBitmap, iris-mpc-gpu/src/dot/kernel.cu:284-349).

The library's comparators keep bitmaps in u32 words with a row stride of
ceil(max_db_length / 64) * 2 words; the bitmap built here has that layout.
On a sharded DB (irisb200.shard) each rank holds entries g % world == rank at
local index g // world, and shard_or_policy_bitmap keeps the bits of one shard
at their local positions.
"""
from __future__ import annotations

import numpy as np


def row_words(max_db_length: int) -> int:
    """u32 words per query row of a comparator bitmap."""
    return (max_db_length + 63) // 64 * 2


def prepare_or_policy_bitmap(max_db_size: int, or_rule_indices, batch_size: int) -> np.ndarray:
    """[batch_size][row_words] u32: bit e of row q is set when DB entry e
    follows the OR rule for query q (prepare_or_policy_bitmap,
    actor.rs:3601-3621)."""
    w = row_words(max_db_size)
    bitmap = np.zeros((batch_size, w), np.uint32)
    for q, ids in enumerate(or_rule_indices):
        for e in ids:
            e = int(e)
            if not 0 <= e < max_db_size:
                raise ValueError(f"OR-rule entry {e} outside the DB")
            bitmap[q, e // 32] |= np.uint32(1 << (e % 32))
    return bitmap


def generate_luc_records(latest_luc_index: int, or_rule_indices, lookback_records: int, batch_size: int,
                         skip_lookback_requests=()) -> list:
    """Per-query OR-rule entries extended with the lookback window
    [latest - lookback, latest] (generate_luc_records, actor.rs:3623-3660):
    with no lookback the input is returned as is; with no OR rules every
    query gets the window; otherwise each query not in
    skip_lookback_requests gets its entries and the window, sorted and
    deduplicated."""
    if lookback_records == 0:
        return [list(x) for x in or_rule_indices]
    start = max(0, latest_luc_index - lookback_records)
    window = list(range(start, latest_luc_index + 1))
    if len(or_rule_indices) == 0:
        return [list(window) for _ in range(batch_size)]
    skip = set(skip_lookback_requests)
    out = []
    for q, ids in enumerate(or_rule_indices):
        ids = list(ids)
        if q not in skip:
            ids = sorted(set(ids) | set(window))
        out.append(ids)
    return out


def shard_or_policy_bitmap(global_bitmap: np.ndarray, max_db_size: int, rank: int, world: int,
                           shard_max_db: int) -> np.ndarray:
    """The bits of one shard of a global OR-policy bitmap at their local
    positions (the reference reads the global bitmap at
    dbIdx * numDevices + deviceId, kernel.cu:326-333)."""
    bits = np.unpackbits(global_bitmap.view(np.uint8), axis=1, bitorder="little")[:, :max_db_size]
    local = bits[:, rank::world]
    n = min(local.shape[1], shard_max_db)
    out = np.zeros((global_bitmap.shape[0], row_words(shard_max_db) * 32), np.uint8)
    out[:, :n] = local[:, :n]
    return np.packbits(out, axis=1, bitorder="little").view(np.uint32)
