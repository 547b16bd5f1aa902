"""The subset pass of the two-stage uniqueness check.

The reference scans the whole DB of one eye at the prefilter ratio 0.375
(THRESHOLD_ANON_STATS_A), collects the matched entries of the batch, and then
re-checks the batch against only those entries at the match ratio 0.345
(THRESHOLD_A), for that eye and for the other eye
(compare_query_against_db_subset_and_self, iris-mpc-gpu/src/server/actor.rs:
1900-2244, called at 1009 and 1076).  The subset is copied out of the resident
DB (prefetch_subset, iris-mpc-gpu/src/dot/share_db.rs:344-407) in chunks of at
most DB_CHUNK_SIZE records, and opened results are mapped back from subset
positions to DB indices (open_subset_results / openResultsWithIndexMapping,
iris-mpc-gpu/src/dot/kernel.cu:118-151).

Here the subset is gathered device-to-device into a small engine per party
(irs_sharedb_gather_records), the batch runs in 32-row slots against it, and
the compacted match lists (irs_dc_take_rows) are mapped back through the id
list on the host.
"""
from __future__ import annotations

import numpy as np

from . import IRIS_CODE_LENGTH, MASK_CODE_LENGTH, MAX_MATCHES_LEN, DistanceComparator, ShareDB, dot_many

DB_CHUNK_SIZE = 32768  # iris-mpc-gpu/src/server/actor.rs:115
MULTS = [1, 1, 1, 2, 2, 2]


class SubsetPass:
    """Re-checks up to `max_queries` queries (31 rotations each) against a
    gathered subset of the DB held by code_engines / mask_engines."""

    def __init__(self, dm, code_engines, mask_engines, circuits, max_queries: int = 64,
                 max_subset: int = DB_CHUNK_SIZE, seeds=None):
        self.dm = dm
        self.ce, self.me = list(code_engines), list(mask_engines)
        self.c = circuits
        self.max_queries = max_queries
        self.max_subset = max_subset
        seeds = seeds or [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]
        rows = max_queries * 32
        self.sce = [ShareDB(p, dm, max_subset, rows, IRIS_CODE_LENGTH, seeds[p]) for p in range(3)]
        self.sme = [ShareDB(p, dm, max_subset, rows, MASK_CODE_LENGTH, seeds[p]) for p in range(3)]
        for e in self.sce + self.sme:
            e.alloc_db(max_subset)
        self.dc = DistanceComparator(dm, max_queries, max(max_subset, 64), match_list_cap=1 << 12)

    def run(self, code_base: np.ndarray, mask_base: np.ndarray, ids, threshold_a: int):
        """code_base [3][nq][12800] / mask_base [3][nq][6400]: the batch's
        preprocessed base shares; ids: DB indices of the subset.  Returns, per
        query, the sorted DB indices it matches among `ids` (at most
        MAX_MATCHES_LEN per subset chunk, as the reference's lists)."""
        nq = code_base.shape[1]
        if nq > self.max_queries:
            raise ValueError("too many queries for this subset pass")
        ids = np.unique(np.asarray(ids, np.int64)).astype(np.uint32)
        out = [[] for _ in range(nq)]
        if ids.size == 0:
            return out
        slots = [(j, 0, 31, j) for j in range(nq)]
        for p in range(3):
            self.sce[p].query_upload_slots(code_base[p], slots)
            self.sme[p].query_upload_slots(mask_base[p], slots)
        for start in range(0, ids.size, self.max_subset):
            chunk = ids[start:start + self.max_subset]
            n = chunk.size
            for p in range(3):
                self.sce[p].gather_records(self.ce[p], chunk)
                self.sme[p].gather_records(self.me[p], chunk)
            self.dc.reset()
            dot_many(self.sce + self.sme, MULTS, 0, n)
            self.dc.compare_threshold_open(self.c, self.sce, self.sme, 0, n, nq, threshold_a)
            counts, pos = self.dc.take_rows(np.arange(nq, dtype=np.uint32), n, clear=True)
            for q in range(nq):
                k = min(int(counts[q]), MAX_MATCHES_LEN)
                out[q].extend(chunk[pos[q, :k]].tolist())  # subset position -> DB index
        return [sorted(x) for x in out]

    def close(self) -> None:
        for o in self.sce + self.sme + [self.dc]:
            o.close()
