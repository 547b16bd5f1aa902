"""Writes into the resident DB between batches: an identity update (a new
record written at an index, write_db_at_index, actor.rs:3547-3600) becomes
matchable, and a deletion (the default-iris record, actor.rs:2641-2680)
removes a match; each pass equals the CPU path on the records read back."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
import workload as W

pytestmark = pytest.mark.gpu

N_DB, NQ, A = 512, 4, 16384


def _scan(dm, c, ce, me, qc, qm):
    dc = irisb200.DistanceComparator(dm, NQ, N_DB)
    try:
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, N_DB)
        dc.compare_threshold_open(c, ce, me, 0, N_DB, NQ, A)
        dm.synchronize()
        return irisb200.bitmap_get(dc.fetch_bitmap(NQ, N_DB), NQ, N_DB)
    finally:
        dc.close()


def test_update_and_delete(dm, oracle):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, 0xAB12)
    qc, qm, plain = W.make_queries(oracle, NQ, codes, masks, 9, {0: (100, 0), 2: (300, 5)})
    ce = [irisb200.ShareDB(p, dm, N_DB, NQ * 32, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, N_DB, NQ * 32, 6400, W.SEEDS[p]) for p in range(3)]
    c = irisb200.Circuits(dm, W.SEEDS)
    slots = [(j, 0, 31, j) for j in range(NQ)]
    try:
        for p in range(3):
            ce[p].alloc_db(N_DB)
            me[p].alloc_db(N_DB)
            ce[p].load_records(0, cs[p])
            me[p].load_records(0, ms[p])
            ce[p].query_upload_slots(qc[p], slots)
            me[p].query_upload_slots(qm[p], slots)
        before = _scan(dm, c, ce, me, qc, qm)
        assert before[0, 100] and before[2, 300]
        # identity update: entry 7 becomes query 1's own iris (fresh shares)
        code1, mask1 = plain[1]
        rc, rm = irisb200.encode_iris(code1, mask1, seed=777)
        for p in range(3):
            ce[p].load_records(7, rc[p][None])
            me[p].load_records(7, rm[p][None])
        # deletion of entry 100
        irisb200.delete_records(ce, me, [100])
        after = _scan(dm, c, ce, me, qc, qm)
        assert after[1, 7] and not after[0, 100] and after[2, 300]
        cs2 = np.stack([ce[p].fetch_records(0, N_DB) for p in range(3)])
        ms2 = np.stack([me[p].fetch_records(0, N_DB) for p in range(3)])
        assert np.array_equal(after, W.expected_bitmap(oracle, qc, qm, cs2, ms2, A))
        assert not after[:, 100].any()  # the deletion record matches none of the queries
    finally:
        c.close()
        for e in ce + me:
            e.close()
