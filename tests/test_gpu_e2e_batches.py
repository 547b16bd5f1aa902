"""Multi-batch run of the plain uniqueness path with insertions, as the
reference's GPU end-to-end test drives its actors (iris-mpc-gpu/tests/e2e.rs:39-271,
TestCaseGenerator::run_n_batches in iris-mpc-common/src/test.rs): per batch
the queries are scanned against the DB in chunks and against the batch
itself, the results merged (smallest matched DB id, in-batch duplicate, or no
match; mergeDbResults / mergeBatchResults), the record assembled
(irisb200.job.assemble_job_result: insertion indices, actor.rs:3197-3303), and
every unique query written into the DB at its insertion index, so that later
batches must find it.  Each batch's final results, counters and insertion
indices must equal the CPU path over the DB as it stood before the batch.
"""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
import workload as W
from irisb200.job import NON_MATCH_ID, BatchInfo, PassOutput, assemble_job_result

pytestmark = pytest.mark.gpu

N_DB0 = 2048
BATCH = 32
N_BATCHES = 6
CAP = N_DB0 + N_BATCHES * BATCH
A = 16384
MULTS = [1, 1, 1, 2, 2, 2]


def _engines(dm, n_db, n_rows):
    ce = [irisb200.ShareDB(p, dm, n_db, n_rows, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, n_db, n_rows, 6400, W.SEEDS[p]) for p in range(3)]
    for e in ce + me:
        e.alloc_db(n_db)
    return ce, me


def _batch_queries(oracle, rng, b, plain_db, n_base, n_db):
    """32 plaintext queries: near-duplicates of base DB entries, of entries
    inserted by earlier batches, exact rotated repeats of an earlier query of
    the same batch, and fresh irises.  Returns [(code, mask)] and the kinds."""
    out, kinds = [], []
    for j in range(BATCH):
        r = int(rng.integers(-15, 16))
        pick = rng.random()
        if pick < 0.25:
            e = int(rng.integers(0, n_base))
            code = oracle.iris_flip(1000 + b, j, 0.1, plain_db[e][0])
            c, m, kind = oracle.iris_rotate(code, r), oracle.iris_rotate(plain_db[e][1], r), "db"
        elif pick < 0.40 and n_db > n_base:
            e = int(rng.integers(n_base, n_db))
            code = oracle.iris_flip(2000 + b, j, 0.1, plain_db[e][0])
            c, m, kind = oracle.iris_rotate(code, r), oracle.iris_rotate(plain_db[e][1], r), "inserted"
        elif pick < 0.55 and j > 0:
            src = out[int(rng.integers(0, j))]
            c, m, kind = oracle.iris_rotate(src[0], r), oracle.iris_rotate(src[1], r), "peer"
        else:
            c, m = oracle.iris_random(3000 + b, j)
            kind = "fresh"
        out.append((c, m))
        kinds.append(kind)
    return out, kinds


def test_batches_with_insertions_match_cpu(dm, oracle):
    rng = np.random.default_rng(2024)
    codes, masks, cs, ms = W.make_db(oracle, N_DB0, 0xDEADBEEF)
    plain_db = list(zip(codes, masks))
    db_cs = np.zeros((3, CAP, 12800), np.uint16)
    db_ms = np.zeros((3, CAP, 6400), np.uint16)
    db_cs[:, :N_DB0], db_ms[:, :N_DB0] = cs, ms
    db_len = N_DB0
    n_rows = BATCH * 32
    ce, me = _engines(dm, CAP, n_rows)
    bce, bme = _engines(dm, BATCH, n_rows)  # the batch as a DB, for the self check
    c = irisb200.Circuits(dm, W.SEEDS)
    dc = irisb200.DistanceComparator(dm, BATCH, CAP)
    slots = [(j, 0, 31, j) for j in range(BATCH)]
    seen = {"db": 0, "inserted": 0, "peer": 0}
    try:
        for p in range(3):
            ce[p].load_records(0, cs[p])
            me[p].load_records(0, ms[p])
        for b in range(N_BATCHES):
            queries, kinds = _batch_queries(oracle, rng, b, plain_db, N_DB0, db_len)
            qc = np.zeros((3, BATCH, 12800), np.uint16)
            qm = np.zeros((3, BATCH, 6400), np.uint16)
            bc = np.zeros((3, BATCH, 12800), np.uint16)  # DB-format shares of the batch
            bm = np.zeros((3, BATCH, 6400), np.uint16)
            for j, (code, mask) in enumerate(queries):
                s = int(oracle.lib().orc_rng64(0x5151 + b, j))
                bc[:, j] = oracle.encode_iris_code(code, mask, s)
                bm[:, j] = oracle.encode_mask_code(mask, s)
                for p in range(3):
                    qc[p, j] = oracle.preprocess_query(p, bc[p, j])
                    qm[p, j] = oracle.preprocess_query(p, bm[p, j])
            for p in range(3):
                for e in (ce[p], bce[p]):
                    e.query_upload_slots(qc[p], slots)
                for e in (me[p], bme[p]):
                    e.query_upload_slots(qm[p], slots)
                bce[p].load_records(0, bc[p])
                bme[p].load_records(0, bm[p])
            for e in ce + me + bce + bme:
                e.set_batch(b + 1)
            c.set_batch(b + 1)
            dc.reset()
            # the DB in two chunks, then the batch against itself
            half = (db_len // 2 + 31) // 32 * 32
            for off, ln in ((0, half), (half, db_len - half)):
                irisb200.dot_many(ce + me, MULTS, off, ln)
                dc.compare_threshold_open(c, ce, me, off, ln, BATCH, A)
            irisb200.dot_many(bce + bme, MULTS, 0, BATCH)
            dc.compare_threshold_open(c, bce, bme, 0, BATCH, BATCH, A, self_check=True)
            dc.join_db_matches(BATCH, db_len)
            dc.join_batch_matches(BATCH)
            final, counters, allm = dc.fetch_final_results(BATCH)

            # the CPU path over the DB as it stood, and over the batch
            exp_db = W.expected_bitmap(oracle, qc, qm, db_cs[:, :db_len], db_ms[:, :db_len], A)
            exp_self = W.expected_bitmap(oracle, qc, qm, bc, bm, A)
            for q in range(BATCH):
                hits = np.nonzero(exp_db[q])[0]
                peers = [j for j in range(q) if exp_self[q, j]]
                want = hits.min() if hits.size else (0xFFFFFFFE if peers else NON_MATCH_ID)
                assert final[q] == want, f"batch {b} query {q} ({kinds[q]})"
                assert counters[q] == hits.size + len(peers), f"batch {b} query {q} counter"
                if hits.size and kinds[q] in ("db", "inserted"):
                    seen[kinds[q]] += 1
                elif not hits.size and peers:
                    seen["peer"] += 1

            # the actor's record: unique queries get the next DB indices
            rec = assemble_job_result(BatchInfo([f"r{b}-{j}" for j in range(BATCH)], ["uniqueness"] * BATCH),
                                      PassOutput(final, counters, allm), [db_len], BATCH)
            new = [q for q in range(BATCH) if not rec.matches[q]]
            assert new == [q for q in range(BATCH) if final[q] == NON_MATCH_ID]
            assert [rec.merged_results[q] for q in new] == list(range(db_len, db_len + len(new)))
            # write the inserted entries (DB-format shares) and grow the DB
            if new:
                for p in range(3):
                    ce[p].load_records(db_len, np.ascontiguousarray(bc[p, new]))
                    me[p].load_records(db_len, np.ascontiguousarray(bm[p, new]))
                db_cs[:, db_len:db_len + len(new)] = bc[:, new]
                db_ms[:, db_len:db_len + len(new)] = bm[:, new]
                plain_db.extend(queries[q] for q in new)
                db_len += len(new)
        # the mix exercised every path: DB matches, matches of inserted
        # entries from earlier batches, and in-batch duplicates
        assert seen["db"] > 0 and seen["inserted"] > 0 and seen["peer"] > 0, seen
        assert db_len > N_DB0
    finally:
        for o in ce + me + bce + bme + [c, dc]:
            o.close()
