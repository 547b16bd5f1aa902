"""Distance capture for anonymised statistics (openResults' match distance
buffers, iris-mpc-gpu/src/dot/kernel.cu:73-106): on the prefilter pass every
opened per-rotation match records the DB entry, the query row and the three
parties' additive components of the code and (x2) mask dots.  The recorded
(entry, row) set must equal the per-rotation matches of the CPU path, and the
components must reconstruct the CPU dot products."""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
import workload as W

pytestmark = pytest.mark.gpu

N_DB, NQ, A = 600, 4, irisb200.THRESHOLD_ANON_STATS_A


def test_distance_capture(dm, oracle):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, 0xD15)
    qc, qm, _ = W.make_queries(oracle, NQ, codes, masks, 41, {0: (3, 0), 1: (599, 5), 3: (100, -7)})
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
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, NQ, N_DB)
    try:
        dc.enable_distance_capture(4096)
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, N_DB)
        dc.compare_threshold_open(c, ce, me, 0, N_DB, NQ, A)
        entry, row, code, mask, total = dc.fetch_distances()
        # CPU: per (query row, entry) dots and the match predicate
        expected = {}
        for q in range(NQ):
            rc = [W.rotated_rows(oracle, qc[p][q:q + 1]) for p in range(3)]
            rm = [W.rotated_rows(oracle, qm[p][q:q + 1]) for p in range(3)]
            cd = sum(oracle.dot_u16(rc[p], cs[p]).astype(np.uint64) for p in range(3)) % 65536
            md = sum(2 * oracle.dot_u16(rm[p], ms[p]).astype(np.uint64) for p in range(3)) % 65536
            hit = oracle.match_predicate(cd, md, A)
            for r, e in zip(*np.nonzero(hit)):
                expected[(int(e), q * 32 + int(r))] = (int(cd[r, e]), int(md[r, e]))
        assert total == len(expected) and len(entry) == total
        got = {}
        for i in range(total):
            got[(int(entry[i]), int(row[i]))] = (int(code[:, i].astype(np.uint64).sum() % 65536),
                                                 int(mask[:, i].astype(np.uint64).sum() % 65536))
        assert got == expected
        assert any(e == 3 and r // 32 == 0 for e, r in got) and any(e == 599 for e, _ in got)
        # the capture is reset by the fetch; a second pass appends afresh
        dc.reset()
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, N_DB)
        dc.compare_threshold_open(c, ce, me, 0, N_DB, NQ, A)
        assert dc.fetch_distances(cap=2)[4] == total
    finally:
        dc.close()
        c.close()
        for e in ce + me:
            e.close()


def test_forced_distance_records(dm, oracle):
    """Pairs listed with irs_dc_set_forced_distances (the reference's
    anon_stats_idx: reauth targets) are recorded on every valid row, match or
    not, each row once even when it also matches."""
    codes, masks, cs, ms = W.make_db(oracle, N_DB, 0xD16)
    qc, qm, _ = W.make_queries(oracle, NQ, codes, masks, 43, {0: (3, 0)})
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
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, NQ, N_DB)
    try:
        dc.enable_distance_capture(4096)
        forced = [(2, 50), (0, 3), (3, 599)]
        dc.set_forced_distances(forced)
        irisb200.dot_many(ce + me, [1, 1, 1, 2, 2, 2], 0, N_DB)
        dc.compare_threshold_open(c, ce, me, 0, N_DB, NQ, A)
        entry, row, code, mask, total = dc.fetch_distances()
        expected = {}
        for q in range(NQ):
            rc = [W.rotated_rows(oracle, qc[p][q:q + 1]) for p in range(3)]
            rm = [W.rotated_rows(oracle, qm[p][q:q + 1]) for p in range(3)]
            cd = sum(oracle.dot_u16(rc[p], cs[p]).astype(np.uint64) for p in range(3)) % 65536
            md = sum(2 * oracle.dot_u16(rm[p], ms[p]).astype(np.uint64) for p in range(3)) % 65536
            keep = oracle.match_predicate(cd, md, A).astype(bool)
            for fq, fe in forced:
                if fq == q:
                    keep[:, fe] = True  # all 31 rotation rows of the slot
            for r, e in zip(*np.nonzero(keep)):
                expected[(int(e), q * 32 + int(r))] = (int(cd[r, e]), int(md[r, e]))
        got = {(int(entry[i]), int(row[i])): (int(code[:, i].astype(np.uint64).sum() % 65536),
                                              int(mask[:, i].astype(np.uint64).sum() % 65536))
               for i in range(total)}
        assert total == len(got) == len(expected)
        assert got == expected
        assert sum(1 for e, r in got if e == 50 and r // 32 == 2) == 31
        dc.set_forced_distances([])
    finally:
        dc.close()
        c.close()
        for e in ce + me:
            e.close()
