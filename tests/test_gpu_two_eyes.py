"""Two-eye merge with the OR-policy bitmap (mergeDbResultsWithOrPolicyBitmap,
iris-mpc-gpu/src/dot/kernel.cu:284-349; join_db_matches,
distance_comparator.rs:688-729): left and right eyes are scanned by their own
engines into their own comparators; the merge keeps an entry for a query when
both eyes match it, or when either does and the policy bit of (query, entry)
is set.  Final result = the smallest kept entry, counters and match lists as
the reference's.  Checked bit-exactly against the CPU path of each eye."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
from irisb200.policy import prepare_or_policy_bitmap
import workload as W

pytestmark = pytest.mark.gpu

N_DB, NQ, A = 700, 8, 16384


def _eye(dm, oracle, db_seed, q_seed, planted):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, db_seed)
    qc, qm, _ = W.make_queries(oracle, NQ, codes, masks, q_seed, planted)
    ce = [irisb200.ShareDB(p, dm, N_DB, NQ * 32, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, N_DB, NQ * 32, 6400, W.SEEDS[p]) for p in range(3)]
    slots = [(j, 0, 31, j) for j in range(NQ)]
    for p in range(3):
        ce[p].alloc_db(N_DB)
        me[p].alloc_db(N_DB)
        ce[p].load_records(0, cs[p])
        me[p].load_records(0, ms[p])
        ce[p].query_upload_slots(qc[p], slots)
        me[p].query_upload_slots(qm[p], slots)
    expected = W.expected_bitmap(oracle, qc, qm, cs, ms, A)
    return ce, me, expected


def test_two_eyes_or_policy(dm, oracle):
    left = _eye(dm, oracle, 0x1EF7, 21, {0: (5, 0), 1: (100, 2), 2: (300, -1), 3: (650, 0)})
    right = _eye(dm, oracle, 0x5167, 22, {0: (5, 0), 1: (200, 0), 2: (300, 3), 4: (650, 1)})
    c = irisb200.Circuits(dm, W.SEEDS)
    dcs = [irisb200.DistanceComparator(dm, NQ, N_DB) for _ in range(2)]
    # OR rule for (1, 100), (3, 650), (2, 300) (prepare_or_policy_bitmap)
    policy = prepare_or_policy_bitmap(N_DB, [[], [100], [300], [650]], NQ)
    dpol = irisb200.DeviceBuffer.from_array(dm, policy)
    try:
        for (ce, me, _), dc in zip((left, right), dcs):
            irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, N_DB)
            dc.compare_threshold_open(c, ce, me, 0, N_DB, NQ, A)
        dcs[0].join_db_matches(NQ, N_DB, right=dcs[1], or_policy=dpol.ptr)
        final, counters, allm = dcs[0].fetch_final_results(NQ)
        bl, br = left[2], right[2]
        pol = np.unpackbits(policy.view(np.uint8), axis=1, bitorder="little")[:, :N_DB].astype(bool)
        keep = np.where(pol, bl | br, bl & br)
        for q in range(NQ):
            hits = np.nonzero(keep[q])[0]
            assert int(counters[q]) == hits.size, f"query {q}"
            assert int(final[q]) == (int(hits[0]) if hits.size else 0xFFFFFFFF)
            assert sorted(allm[q, : min(hits.size, 256)].tolist()) == hits[:256].tolist()
        # both eyes: 0 -> 5 and 2 -> 300; policy OR: 1 -> 100 (left only), 3 -> 650 (left only);
        # 4 matches its right eye only, without a policy bit: no match
        assert final[0] == 5 and final[2] == 300 and final[1] == 100 and final[3] == 650
        assert final[4] == 0xFFFFFFFF
        # single eye (no right comparator): the left bitmap alone
        for dc in dcs:
            dc.reset()
        irisb200.dot_many(left[0] + left[1], [1, 1, 1, 2, 2, 2], 0, N_DB)
        dcs[0].compare_threshold_open(c, left[0], left[1], 0, N_DB, NQ, A)
        dcs[0].join_db_matches(NQ, N_DB)
        final1, counters1, _ = dcs[0].fetch_final_results(NQ)
        for q in range(NQ):
            hits = np.nonzero(bl[q])[0]
            assert int(counters1[q]) == hits.size
            assert int(final1[q]) == (int(hits[0]) if hits.size else 0xFFFFFFFF)
    finally:
        dpol.free()
        for dc in dcs:
            dc.close()
        c.close()
        for e in left[0] + left[1] + right[0] + right[1]:
            e.close()
