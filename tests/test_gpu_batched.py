"""Batched uneven launches (dense row packing, reauth subsets, CUDA graphs).

A batch mixes uniqueness and reauth requests with 1, 16 or 31 centred
rotations, half of them with a mirrored variant.  Every request's matches must
equal the CPU path (per-party dots of the variant's rotation rows against the
DB, summed, thresholded, OR over the rows); replaying the captured graph for a
second batch (fresh ChaCha batch id) must give the same revealed results.
"""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
from irisb200.batched import BatchedEngine, Request, centred_rotations
import workload as W

pytestmark = pytest.mark.gpu

N_DB = 1024
A = 20316


@pytest.fixture(scope="module")
def setup(dm, oracle):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, 0xBEEF)
    planted = {0: (5, 2), 2: (700, -9), 3: (64, 15), 6: (1000, 0), 8: (333, -3)}
    qc, qm, _ = W.make_queries(oracle, 10, codes, masks, 99, planted)
    ce = [irisb200.ShareDB(p, dm, N_DB, 2048, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, N_DB, 2048, 6400, W.SEEDS[p]) for p in range(3)]
    for p in range(3):
        ce[p].alloc_db(N_DB)
        me[p].alloc_db(N_DB)
        ce[p].load_records(0, cs[p])
        me[p].load_records(0, ms[p])
    yield dict(codes=codes, masks=masks, cs=cs, ms=ms, qc=qc, qm=qm, ce=ce, me=me, planted=planted)
    for e in ce + me:
        e.close()


def expected_hits(oracle, cs, ms, qc, qm, n_rot, mirrored, entries):
    base_c = [oracle.mirror_share(qc[p], True) if mirrored else qc[p] for p in range(3)]
    base_m = [oracle.mirror_share(qm[p], False) if mirrored else qm[p] for p in range(3)]
    rots = list(centred_rotations(n_rot))
    code = 0
    mask = 0
    for p in range(3):
        rc = np.stack([oracle.rotate_share(base_c[p], r) for r in rots])
        rm = np.stack([oracle.rotate_share(base_m[p], r) for r in rots])
        code = code + oracle.dot_u16(rc, cs[p][entries]).astype(np.uint64)
        mask = mask + 2 * oracle.dot_u16(rm, ms[p][entries]).astype(np.uint64)
    hit = oracle.match_predicate(code % 65536, mask % 65536, A).max(axis=0)
    return [int(e) for e, h in zip(entries, hit) if h]


def test_batched_uneven_mixed_batch(dm, oracle, setup):
    s = setup
    c = irisb200.Circuits(dm, W.SEEDS)
    eng = BatchedEngine(dm, s["ce"], s["me"], c, max_variants=64, max_reauth=16, threshold_a=A)
    try:
        spec = [  # (query, n_rot, mirrored, kind, target)
            (0, 31, False, "uniqueness", -1), (1, 16, True, "uniqueness", -1), (2, 1, False, "uniqueness", -1),
            (3, 31, True, "uniqueness", -1), (4, 1, True, "uniqueness", -1), (5, 16, False, "uniqueness", -1),
            (6, 31, False, "reauth", 1000), (7, 16, True, "reauth", 12), (8, 1, False, "reauth", 333),
            (2, 16, False, "reauth", 700), (9, 31, True, "uniqueness", -1),
        ]
        reqs = [Request(code=s["qc"][:, q], mask=s["qm"][:, q], n_rot=n, mirrored=mir, kind=k, target=t)
                for q, n, mir, k, t in spec]
        for rep in range(2):  # second batch replays the captured graph with a new batch id
            res = eng.run(reqs)
            for (q, n, mir, k, t), r in zip(spec, res):
                qc, qm = s["qc"][:, q], s["qm"][:, q]
                if k == "uniqueness":
                    assert r.matches == expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, False, np.arange(N_DB))
                    if mir:
                        assert r.mirror_matches == expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, True,
                                                                 np.arange(N_DB))
                else:
                    exp = expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, False, np.array([t]))
                    assert r.reauth_match == bool(exp), f"reauth {q}->{t}"
                    if mir:
                        expm = expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, True, np.array([t]))
                        assert r.reauth_mirror_match == bool(expm)
        # planted near-duplicates are found with their centred rotations
        assert 5 in res[0].matches and 64 in res[3].matches
        # query 6 is planted from its target with no shift (31 rotations cover it);
        # queries 8 and 2 were shifted by -3 / -9 columns, which 1 / 16 centred
        # rotations do not cover (checked against the CPU path above)
        assert res[6].reauth_match is True
        assert res[8].reauth_match is False and res[9].reauth_match is False
        assert eng.graphs, "the DB pass must run from a captured graph"
    finally:
        eng.close()
        c.close()


def test_batched_equals_plain_slots(dm, oracle, setup):
    """All-31-rotation uniqueness batch: the batched engine and the plain
    slot path give the same bitmap rows."""
    s = setup
    c = irisb200.Circuits(dm, W.SEEDS)
    eng = BatchedEngine(dm, s["ce"], s["me"], c, max_variants=16, max_reauth=4, threshold_a=A, autotune=False)
    try:
        reqs = [Request(code=s["qc"][:, q], mask=s["qm"][:, q]) for q in range(8)]
        res = eng.run(reqs)
        dc = irisb200.DistanceComparator(dm, 8, N_DB)
        slots = [(j, 0, 31, j) for j in range(8)]
        for p in range(3):
            s["ce"][p].query_upload_slots(s["qc"][p][:8], slots)
            s["me"][p].query_upload_slots(s["qm"][p][:8], slots)
        for e in s["ce"] + s["me"]:
            e.use_batch_counter(False)
            e.set_tile(0)
        c.use_batch_counter(False)
        irisb200.dot_many(s["ce"] + s["me"], [1, 1, 1, 2, 2, 2], 0, N_DB)
        dc.compare_threshold_open(c, s["ce"], s["me"], 0, N_DB, 8, A)
        bm = irisb200.bitmap_get(dc.fetch_bitmap(8, N_DB), 8, N_DB)
        for q in range(8):
            assert res[q].matches == np.nonzero(bm[q])[0].tolist()
        dc.close()
    finally:
        eng.close()
        c.close()


def test_pipelined_batches_match_one_at_a_time(dm, oracle, setup):
    """Two different batches in flight at once (submit, submit, collect,
    collect, and a third submit that collects the batch whose buffers it
    reuses) give the same results as the same batches run one at a time."""
    s = setup
    c = irisb200.Circuits(dm, W.SEEDS)
    eng = BatchedEngine(dm, s["ce"], s["me"], c, max_variants=32, max_reauth=8, threshold_a=A)
    try:
        def req(q, n, mir, k="uniqueness", t=-1):
            return Request(code=s["qc"][:, q], mask=s["qm"][:, q], n_rot=n, mirrored=mir, kind=k, target=t)
        batch_a = [req(0, 31, True), req(3, 16, False), req(6, 31, False, "reauth", 1000), req(1, 1, True)]
        batch_b = [req(3, 31, True), req(8, 1, False, "reauth", 333), req(2, 31, False), req(5, 16, True),
                   req(0, 16, False, "reauth", 5)]
        alone_a, alone_b = eng.run(batch_a), eng.run(batch_b)
        ta, tb = eng.submit(batch_a), eng.submit(batch_b)
        tc = eng.submit(batch_a)  # reuses batch a's buffers: collects it first
        assert ta.results is not None
        for got, want in ((eng.collect(ta), alone_a), (eng.collect(tb), alone_b), (eng.collect(tc), alone_a)):
            assert got == want
        assert 5 in alone_a[0].matches and 64 in alone_b[0].matches
        assert alone_a[2].reauth_match is True
    finally:
        eng.close()
        c.close()


@pytest.mark.parametrize("path", ["split", "pair", "fused"])
def test_batched_every_tuner_candidate(dm, oracle, setup, path):
    """Every (path, tile, chunk) candidate the autotuner may pick gives the CPU
    path's matches: the GEMM launch + threshold launch at each tile width, the
    two-SM GEMM, and the one-kernel fused scan; and each path's captured pass
    over several chunks with a ragged last one (1024 = 2 x 384 + 256)."""
    s = setup
    c = irisb200.Circuits(dm, W.SEEDS)
    eng = BatchedEngine(dm, s["ce"], s["me"], c, max_variants=64, max_reauth=16, threshold_a=A, autotune=False,
                        path=path)
    try:
        spec = [(0, 31, False, "uniqueness", -1), (1, 16, True, "uniqueness", -1), (3, 31, True, "uniqueness", -1),
                (4, 1, True, "uniqueness", -1), (6, 31, False, "reauth", 1000), (9, 31, True, "uniqueness", -1),
                (8, 16, False, "uniqueness", -1)]
        reqs = [Request(code=s["qc"][:, q], mask=s["qm"][:, q], n_rot=n, mirrored=mir, kind=k, target=t)
                for q, n, mir, k, t in spec]
        eng.run(reqs)  # fixes the padded row count the tuner keys on
        (n_pad, first), = eng.tuned.items()
        assert first[0] == path
        cands = [cd for cd in BatchedEngine._candidates(n_pad, N_DB) if cd[0] == path]
        assert cands
        cands += sorted({(p, t, 384) for p, t, _ in cands})
        for cand in cands:
            eng.tuned = {n_pad: cand}
            res = eng.run(reqs)
            for (q, n, mir, k, t), r in zip(spec, res):
                qc, qm = s["qc"][:, q], s["qm"][:, q]
                if k == "uniqueness":
                    assert r.matches == expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, False, np.arange(N_DB)), \
                        f"{cand} query {q}"
                    if mir:
                        assert r.mirror_matches == expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, True,
                                                                 np.arange(N_DB)), f"{cand} mirrored query {q}"
                else:
                    exp = expected_hits(oracle, s["cs"], s["ms"], qc, qm, n, False, np.array([t]))
                    assert r.reauth_match == bool(exp), f"{cand} reauth {q}->{t}"
    finally:
        eng.close()
        c.close()
