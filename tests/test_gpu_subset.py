"""Two-stage check: a full scan at the prefilter ratio 0.375 collects the
batch's candidates, the subset pass re-checks the batch against only those
entries at 0.345 (compare_query_against_db_subset_and_self,
iris-mpc-gpu/src/server/actor.rs:1900-2244).  Because every 0.345 match is a
0.375 match, the two-stage result must equal a full scan at 0.345, entry for
entry, and the subset pass on the other eye must equal that eye's full scan
restricted to the same candidates.  Subsets larger than one chunk are split."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
from irisb200.subset import SubsetPass
import workload as W

pytestmark = pytest.mark.gpu

N_DB, NQ = 1500, 8


def _engines(dm, oracle, db_seed, q_seed, planted):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, db_seed)
    qc, qm, _ = W.make_queries(oracle, NQ, codes, masks, q_seed, planted)
    ce = [irisb200.ShareDB(p, dm, N_DB, NQ * 32, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, N_DB, NQ * 32, 6400, W.SEEDS[p]) for p in range(3)]
    for p in range(3):
        ce[p].alloc_db(N_DB)
        me[p].alloc_db(N_DB)
        ce[p].load_records(0, cs[p])
        me[p].load_records(0, ms[p])
    return ce, me, cs, ms, qc, qm


def test_two_stage_equals_full_scan(dm, oracle):
    # planted near-duplicates; 0.2-flip copies match at both ratios, and query 5
    # duplicates entries 40 and 1400 so that several candidates share a query
    left = _engines(dm, oracle, 0xA11CE, 31, {0: (7, 0), 1: (640, 4), 3: (1499, -6), 5: (40, 0), 6: (1400, 1)})
    right = _engines(dm, oracle, 0xB0B, 32, {0: (7, 1), 1: (900, 0), 3: (1499, 0), 6: (1400, -2)})
    c = irisb200.Circuits(dm, W.SEEDS)
    sp_l = SubsetPass(dm, left[0], left[1], c, max_queries=NQ, max_subset=3)  # tiny chunks: exercises splitting
    sp_r = SubsetPass(dm, right[0], right[1], c, max_queries=NQ, max_subset=64)
    try:
        ce, me, cs, ms, qc, qm = left
        # stage 1: full scan of the left eye at the prefilter ratio
        pre = W.expected_bitmap(oracle, qc, qm, cs, ms, irisb200.THRESHOLD_ANON_STATS_A)
        dc = irisb200.DistanceComparator(dm, NQ, N_DB)
        slots = [(j, 0, 31, j) for j in range(NQ)]
        for p in range(3):
            ce[p].query_upload_slots(qc[p], slots)
            me[p].query_upload_slots(qm[p], slots)
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, N_DB)
        dc.compare_threshold_open(c, ce, me, 0, N_DB, NQ, irisb200.THRESHOLD_ANON_STATS_A)
        counts, pos = dc.take_rows(np.arange(NQ, dtype=np.uint32), N_DB)
        cand = sorted({int(e) for q in range(NQ) for e in pos[q, : int(counts[q])]})
        assert cand == sorted(set(np.nonzero(pre.any(axis=0))[0].tolist()))
        dc.close()
        # stage 2: the subset pass at the match ratio, both eyes, same candidates
        got_l = sp_l.run(qc, qm, cand, irisb200.THRESHOLD_A)
        full_l = W.expected_bitmap(oracle, qc, qm, cs, ms, irisb200.THRESHOLD_A)
        for q in range(NQ):
            assert got_l[q] == np.nonzero(full_l[q])[0].tolist(), f"left query {q}"
        _, _, csr, msr, qcr, qmr = right
        got_r = sp_r.run(qcr, qmr, cand, irisb200.THRESHOLD_A)
        full_r = W.expected_bitmap(oracle, qcr, qmr, csr, msr, irisb200.THRESHOLD_A)
        for q in range(NQ):
            assert got_r[q] == [e for e in np.nonzero(full_r[q])[0].tolist() if e in cand], f"right query {q}"
        assert 7 in got_l[0] and 7 in got_r[0] and 1499 in got_l[3] and 1499 in got_r[3]
        assert got_l[2] == [] and sp_l.run(qc, qm, [], irisb200.THRESHOLD_A) == [[] for _ in range(NQ)]
    finally:
        sp_l.close()
        sp_r.close()
        c.close()
        for e in left[0] + left[1] + right[0] + right[1]:
            e.close()


def _rotation_hits(oracle, cs, ms, qc, qm, entries, threshold_a):
    """{entry: sorted signed rotations (-15..15) at which the query matches}
    on the CPU: per-party dots of all 31 rotation rows, summed, thresholded."""
    entries = np.asarray(entries)
    code = 0
    mask = 0
    for p in range(3):
        rc = np.stack([oracle.rotate_share(qc[p], r) for r in range(31)])
        rm = np.stack([oracle.rotate_share(qm[p], r) for r in range(31)])
        code = code + oracle.dot_u16(rc, cs[p][entries]).astype(np.uint64)
        mask = mask + 2 * oracle.dot_u16(rm, ms[p][entries]).astype(np.uint64)
    hit = oracle.match_predicate(code % 65536, mask % 65536, threshold_a)  # [31][n]
    return {int(e): [r - 15 for r in range(31) if hit[r, k]] for k, e in enumerate(entries) if hit[:, k].any()}


def test_subset_rotation_indices(dm, oracle):
    """partial_match_rotation_indices: for every DB index a query matches in
    the subset pass, the signed rotations that matched, == the CPU path.
    Planted copies shifted by r match around rotation -r; a query planted
    twice from one entry covers two DB indices."""
    ce, me, cs, ms, qc, qm = _engines(dm, oracle, 0xC0FFEE, 33, {0: (11, 0), 2: (500, 5), 4: (1200, -7), 7: (11, 3)})
    c = irisb200.Circuits(dm, W.SEEDS)
    sp = SubsetPass(dm, ce, me, c, max_queries=NQ, max_subset=4, rotations=True)
    try:
        cand = [3, 11, 12, 500, 777, 1200, 1499]
        ids, rots = sp.run_with_rotations(qc, qm, cand, irisb200.THRESHOLD_A)
        assert sp.rotations_lost == 0
        for q in range(NQ):
            want = _rotation_hits(oracle, cs, ms, qc[:, q], qm[:, q], cand, irisb200.THRESHOLD_A)
            assert ids[q] == sorted(want), f"query {q}"
            assert rots[q] == [want[e] for e in ids[q]], f"query {q}"
        assert 11 in ids[0] and 500 in ids[2] and 1200 in ids[4] and 11 in ids[7]
        assert all(len(r) >= 1 for q in range(NQ) for r in rots[q])
        assert sp.run(qc, qm, cand, irisb200.THRESHOLD_A) == ids  # run() == the ids of run_with_rotations
        assert sp.match_counts.tolist() == [len(x) for x in ids]  # partial_match_counters
    finally:
        sp.close()
        c.close()
        for e in ce + me:
            e.close()
