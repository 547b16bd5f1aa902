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

The reference also records, for every opened (query rotation, subset entry)
match, the signed rotation (-15..15) next to the DB index
(openResultsWithIndexMapping, kernel.cu:118-151; get_partial_results_with_
rotations, distance_comparator.rs:650-711), and the actor lists the matching
rotations of each partial match (map_rotation_indices_to_db_ids_per_query,
actor.rs:2859-2883).  run_with_rotations does the same from the comparator's
distance capture, whose records carry the query row (32 * query + rotation
index) of each opened match.
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
                 max_subset: int = DB_CHUNK_SIZE, seeds=None, rotations: bool = False):
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
        # rotation records: as the reference, up to MAX_MATCHES_LEN per query row
        self.rot_cap = MAX_MATCHES_LEN * 31 * max_queries if rotations else 0
        self.rotations_lost = 0
        self.match_counts = np.zeros(0, np.int64)
        if rotations:
            self.dc.enable_distance_capture(self.rot_cap)

    def run(self, code_base: np.ndarray, mask_base: np.ndarray, ids, threshold_a: int):
        """code_base [3][nq][12800] / mask_base [3][nq][6400]: the batch's
        preprocessed base shares; ids: DB indices of the subset.  Returns, per
        query, the sorted DB indices it matches among `ids` (at most
        MAX_MATCHES_LEN per subset chunk, as the reference's lists)."""
        return self._run(code_base, mask_base, ids, threshold_a, False)[0]

    def run_with_rotations(self, code_base: np.ndarray, mask_base: np.ndarray, ids, threshold_a: int):
        """run() plus, per query, one sorted list of the matching signed
        rotations (-15..15, 0 = centre) for each returned DB index
        (partial_match_rotation_indices).  Needs rotations=True at
        construction; self.rotations_lost counts records beyond the capture
        capacity (the reference drops them too)."""
        if not self.rot_cap:
            raise ValueError("construct the subset pass with rotations=True")
        return self._run(code_base, mask_base, ids, threshold_a, True)

    def _run(self, code_base, mask_base, ids, threshold_a: int, want_rot: bool):
        nq = code_base.shape[1]
        if nq > self.max_queries:
            raise ValueError("too many queries for this subset pass")
        ids = np.unique(np.asarray(ids, np.int64)).astype(np.uint32)
        out = [[] for _ in range(nq)]
        rot = [dict() for _ in range(nq)]  # query -> DB index -> rotations
        self.rotations_lost = 0
        # partial_match_counters: every match of the query, also those past
        # the MAX_MATCHES_LEN ids a chunk returns
        self.match_counts = np.zeros(nq, np.int64)
        if ids.size == 0:
            return out, [[] for _ in range(nq)]
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
            self.match_counts += counts[:nq].astype(np.int64)
            for q in range(nq):
                k = min(int(counts[q]), MAX_MATCHES_LEN)
                out[q].extend(chunk[pos[q, :k]].tolist())  # subset position -> DB index
            if self.rot_cap:
                entry, row, _, _, total = self.dc.fetch_distances(self.rot_cap, reset=True)
                self.rotations_lost += max(0, total - self.rot_cap)
                if want_rot:
                    for e, r in zip(entry.tolist(), row.tolist()):
                        q, ri = divmod(r, 32)  # slot q holds query q's 31 rotations
                        rot[q].setdefault(int(chunk[e]), []).append(ri - 15)
        out = [sorted(x) for x in out]
        return out, [[sorted(rot[q].get(e, [])) for e in out[q]] for q in range(nq)]

    def close(self) -> None:
        for o in self.sce + self.sme + [self.dc]:
            o.close()
