"""Continuous-batching server: results alone equal results in the mix.

Requests of every kind arrive open-loop while others are scanning: uniqueness
requests with 31, 16 or 1 centred rotations (some mirrored), reauth requests
and an append.  The row capacity is small, so requests queue for rows and are
admitted mid-scan at arbitrary chunk boundaries.  Every uniqueness result must
equal (a) the same request served alone and (b) the CPU path over the DB as it
was when the request was admitted: an append is matched by requests that
arrive after it and by none before.  The DB length is not a multiple of the
chunk (ragged last chunk).
"""
from __future__ import annotations

import numpy as np
import pytest

import irisb200
from irisb200.batched import Request, centred_rotations
from irisb200.serving import ContinuousServer
import workload as W

pytestmark = pytest.mark.gpu

N_DB = 1500
CHUNK = 512
ROWS = 128
A = 20316


@pytest.fixture(scope="module")
def world(dm, oracle):
    codes, masks, cs, ms = W.make_db(oracle, N_DB, 0xC0FFEE)
    xcodes, xmasks, xcs, xms = W.make_db(oracle, 1, 0xABCD)  # the appended iris
    planted = {0: (10, 0), 1: (700, 4), 2: (1499, -2), 3: (512, 0)}
    qc, qm, _ = W.make_queries(oracle, 5, codes, masks, 77, planted)
    xqc, xqm, _ = W.make_queries(oracle, 2, xcodes, xmasks, 78, {0: (0, 0), 1: (0, 1)})
    ce = [irisb200.ShareDB(p, dm, CHUNK, ROWS, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, CHUNK, ROWS, 6400, W.SEEDS[p]) for p in range(3)]
    for p in range(3):
        ce[p].alloc_db(N_DB + 16)
        me[p].alloc_db(N_DB + 16)
        ce[p].load_records(0, cs[p])
        me[p].load_records(0, ms[p])
    c = irisb200.Circuits(dm, W.SEEDS)
    srv = ContinuousServer(dm, ce, me, c, chunk=CHUNK, row_capacity=ROWS, max_variants=32, max_reauth=8,
                           threshold_a=A, db_capacity=N_DB + 16)
    all_cs = np.concatenate([cs, xcs], axis=1)
    all_ms = np.concatenate([ms, xms], axis=1)
    yield dict(qc=qc, qm=qm, xqc=xqc, xqm=xqm, xcs=xcs, xms=xms, cs=all_cs, ms=all_ms, srv=srv)
    srv.close()
    c.close()
    for e in ce + me:
        e.close()


def _requests(w):
    def q(src, j, n_rot=31, mirrored=False, kind="uniqueness", target=-1):
        code, mask = (w["qc"], w["qm"]) if src == "q" else (w["xqc"], w["xqm"])
        return Request(code=code[:, j], mask=mask[:, j], n_rot=n_rot, mirrored=mirrored, kind=kind, target=target)
    return [
        q("q", 0),                                    # 0
        q("q", 1, 16, True),                          # 1
        q("q", 3, 31, False, "reauth", 512),          # 2
        q("x", 0),                                    # 3  before the append: must not match it
        Request(code=None, mask=None, kind="append"),  # 4  appends the iris at index N_DB
        q("q", 2, 1, True),                           # 5
        q("x", 1, 31, True),                          # 6  after the append: matches index N_DB
        q("q", 4),                                    # 7
        q("q", 0, 16, True, "reauth", 10),            # 8
        q("q", 3),                                    # 9
        q("q", 1, 31, True),                          # 10
    ]


def test_serving_alone_equals_mix_and_cpu(oracle, world):
    w = world
    srv = w["srv"]
    reqs = _requests(w)
    uniq = [i for i, r in enumerate(reqs) if r.kind == "uniqueness"]
    # (1) each uniqueness request alone, on the initial DB
    alone = {}
    for i in uniq:
        (comp,) = srv.serve([0.0], [reqs[i]])
        alone[i] = comp.result
        r = reqs[i]
        rots = list(centred_rotations(r.n_rot))
        assert alone[i].matches == W.expected_variant_hits(oracle, w["cs"], w["ms"], r.code, r.mask, rots, False,
                                                           np.arange(N_DB), A), f"request {i} alone"
        if r.mirrored:
            assert alone[i].mirror_matches == W.expected_variant_hits(
                oracle, w["cs"], w["ms"], r.code, r.mask, rots, True, np.arange(N_DB), A), f"request {i} mirror"
    assert 10 in alone[0].matches and 512 in alone[9].matches
    # (2) the mix, open loop: arrivals 1 ms apart, rows for ~3 requests at a time
    arrivals = [0.001 * i for i in range(len(reqs))]
    appends = {4: (w["xcs"][:, 0], w["xms"][:, 0])}
    comps = srv.serve(arrivals, reqs, appends=appends)
    assert sorted(c.idx for c in comps) == list(range(len(reqs)))
    res = {c.idx: c.result for c in comps}
    assert srv.db_len == N_DB + 1
    for i in uniq:
        r = reqs[i]
        snap = N_DB + 1 if i > 4 else N_DB
        rots = list(centred_rotations(r.n_rot))
        exp = W.expected_variant_hits(oracle, w["cs"], w["ms"], r.code, r.mask, rots, False, np.arange(snap), A)
        assert res[i].matches == exp, f"request {i} in the mix"
        assert res[i].matches == alone[i].matches + ([N_DB] if N_DB in exp else []), f"request {i}: alone != mix"
        if r.mirrored:
            expm = W.expected_variant_hits(oracle, w["cs"], w["ms"], r.code, r.mask, rots, True, np.arange(snap), A)
            assert res[i].mirror_matches == expm
    assert N_DB not in res[3].matches          # arrived before the append
    assert N_DB in res[6].matches              # arrived after it
    for i in (2, 8):
        r = reqs[i]
        rots = list(centred_rotations(r.n_rot))
        exp = W.expected_variant_hits(oracle, w["cs"], w["ms"], r.code, r.mask, rots, False, [r.target], A)
        assert res[i].reauth_match == bool(exp)
        if r.mirrored:
            expm = W.expected_variant_hits(oracle, w["cs"], w["ms"], r.code, r.mask, rots, True, [r.target], A)
            assert res[i].reauth_mirror_match == bool(expm)
    assert res[2].reauth_match is True and res[8].reauth_match is True
    assert srv.steps > 0 and not srv.flight and len(srv.free_variants) == 32
    # checkpoint / restore between serve() calls: the ChaCha batch counter and the DB length
    state = srv.checkpoint()
    assert state["db_len"] == N_DB + 1 and state["batch_counter"] >= srv.steps
    srv.restore(state)
    assert srv.dm.batch_counter() == state["batch_counter"] and srv.db_len == N_DB + 1


def test_two_sm_gemm_server_equals_default(dm, oracle, world):
    """With the two-SM GEMM (gemm_pair=True; it applies once the rows in flight
    pad to the 256-row tile: here 30 variants of 31 rotations, 1024 rows) the
    server returns the same matches as with the default GEMM, and the CPU
    path's."""
    cs, ms = world["cs"][:, :N_DB], world["ms"][:, :N_DB]
    rows = 1024
    ce = [irisb200.ShareDB(p, dm, CHUNK, rows, 12800, W.SEEDS[p]) for p in range(3)]
    me = [irisb200.ShareDB(p, dm, CHUNK, rows, 6400, W.SEEDS[p]) for p in range(3)]
    c = irisb200.Circuits(dm, W.SEEDS)
    try:
        for p in range(3):
            ce[p].alloc_db(N_DB)
            me[p].alloc_db(N_DB)
            ce[p].load_records(0, cs[p])
            me[p].load_records(0, ms[p])
        reqs = [Request(code=world["qc"][:, j % 5], mask=world["qm"][:, j % 5], n_rot=31, mirrored=j % 2 == 1)
                for j in range(20)]
        got = {}
        for pair in (False, True):
            srv = ContinuousServer(dm, ce, me, c, chunk=CHUNK, row_capacity=rows, max_variants=32, max_reauth=4,
                                   threshold_a=A, db_capacity=N_DB, gemm_pair=pair)
            try:
                comps = srv.serve([0.0] * len(reqs), reqs)
                assert srv.stats["rows"] >= 1024 * srv.stats["steps"] * 0.5, "the 256-row tile was not reached"
            finally:
                srv.close()
            got[pair] = {cp.idx: (cp.result.matches, cp.result.mirror_matches) for cp in comps}
        assert got[True] == got[False]
        for j in range(5):
            for mir in (False, True):
                exp = W.expected_variant_hits(oracle, cs, ms, world["qc"][:, j], world["qm"][:, j], list(range(31)),
                                              mir, np.arange(N_DB), A)
                i = j if (not mir or j % 2 == 1) else j + 5  # odd requests carry a mirrored variant
                assert got[True][i][1 if mir else 0] == exp[:256], f"query {j} mirrored={mir}"
    finally:
        c.close()
        for e in ce + me:
            e.close()
