"""Sharded DB across ranks (gloo, world size 2, CPU): every rank scans its
round-robin shard (global entry g on rank g % 2, local index g // 2), then one
all_gather merges the results.  The merged first-match index, match counts and
match lists must equal the unsharded scan; reauth targets and appends are
routed to the rank that holds them.  The per-shard scan is the CPU oracle's
plain match (the GPU engine computes the same bitmap bit-exactly)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from irisb200.shard import (NON_MATCH_ID, append_target, exchange_results, global_id, merge_final_results,
                            shard_entries, shard_len, shard_of)

N_DB, NQ, A, CAP = 300, 4, 16384, 256


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _world_data():
    from oracle import oracle as O
    import workload as W
    O.build()
    codes, masks, cs, ms = W.make_db(O, N_DB, 0xABC)
    planted = {0: (17, 0), 1: (250, 3), 3: (18, -2)}
    qc, qm, _ = W.make_queries(O, NQ, codes, masks, 5, planted)
    return O, W, cs, ms, qc, qm


def _scan(O, W, cs, ms, qc, qm, entries):
    bm = W.expected_bitmap(O, qc, qm, cs[:, entries], ms[:, entries], A, 1)
    final = np.full(NQ, NON_MATCH_ID, np.int64)
    counts = np.zeros(NQ, np.int64)
    ids = np.zeros((NQ, CAP), np.int64)
    for q in range(NQ):
        hit = np.nonzero(bm[q])[0]
        counts[q] = hit.size
        if hit.size:
            final[q] = hit[0]
        ids[q, : min(hit.size, CAP)] = hit[:CAP]
    return final, counts, ids, bm


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        O, W, cs, ms, qc, qm = _world_data()
        entries = shard_entries(N_DB, rank, world)
        assert entries.size == shard_len(N_DB, rank, world)
        final, counts, ids, _ = _scan(O, W, cs, ms, qc, qm, entries)
        mf, mc, lists = exchange_results(final, counts, ids)
        out[rank] = (mf.tolist(), mc.tolist(), [x.tolist() for x in lists])
    finally:
        dist.destroy_process_group()


def test_sharded_scan_merges_to_the_unsharded_result():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    O, W, cs, ms, qc, qm = _world_data()
    final, counts, ids, bm = _scan(O, W, cs, ms, qc, qm, np.arange(N_DB))
    for r in range(world):
        mf, mc, lists = res[r]
        assert mf == [int(x) for x in final], "first match"
        assert mc == counts.tolist()
        for q in range(NQ):
            assert lists[q] == np.nonzero(bm[q])[0].tolist()
    assert final[0] == 17 and 250 in res[0][2][1]


def test_routing():
    world = 8
    g = np.arange(1000)
    r, loc = shard_of(g, world)
    assert (global_id(loc, r, world) == g).all()
    assert sum(shard_len(1000, k, world) for k in range(world)) == 1000
    assert append_target(1000, world) == (0, 125) and append_target(1003, world) == (3, 125)
    # per-shard first matches merge to the smallest global index
    assert merge_final_results([[NON_MATCH_ID, 5, 7], [2, NON_MATCH_ID, 3]]).tolist() == \
        [2 * 2 + 1, 5 * 2, 3 * 2 + 1]
