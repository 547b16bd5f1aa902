"""ServerJobResult assembly (host, no GPU) against hand-built expected records.

The rules follow iris-mpc-gpu/src/server/actor.rs: merged results and
insertion indices (1289-1419, calculate_insertion_indices 3270-3303,
distribute_insertions 3197-3210), the supermatcher limit (117), skipped
persistence, batch peers from the dummy ids U32_MAX - j (1422-1453), reauth
success (1463-1475) and the full-face mirror attack flag from the mirror
pass's record (1316-1370)."""
from __future__ import annotations

import numpy as np

from irisb200.batched import Request, Result
from irisb200.job import (NON_MATCH_ID, U32_MAX, BatchInfo, PassOutput, assemble_job_result,
                          calculate_insertion_indices, distribute_insertions, pass_output_from_requests)


def _pass(final, counters, lists, pl=None, pr=None):
    am = np.zeros((len(final), 256), np.uint32)
    for i, ids in enumerate(lists):
        am[i, :len(ids)] = ids
    kw = {}
    if pl is not None:
        kw.update(partial_ids_left=[[] for _ in final], partial_counters_left=pl)
    if pr is not None:
        kw.update(partial_ids_right=[[] for _ in final], partial_counters_right=pr)
    return PassOutput(np.array(final, np.uint32), np.array(counters, np.uint32), am, **kw)


BATCH = BatchInfo(
    request_ids=[f"r{i}" for i in range(7)],
    request_types=["uniqueness", "uniqueness", "reauth", "uniqueness", "uniqueness", "reset_check", "uniqueness"],
    skip_persistence=[False, False, False, False, True, False, False],
    reauth_target_indices={"r2": 77}, reauth_use_or_rule={"r2": False})


def test_single_orientation_record():
    out = _pass(final=[12, NON_MATCH_ID, 77, NON_MATCH_ID - 1, NON_MATCH_ID, NON_MATCH_ID, NON_MATCH_ID],
                counters=[2, 0, 1, 1, 0, 0, 0],
                lists=[[12, 40], [], [77], [U32_MAX - 1], [], [], []],
                pl=[3, 10, 1, 1, 0, 0, 0], pr=[2, 5000, 1, 1, 0, 0, 0])
    r = assemble_job_result(BATCH, out, db_sizes=[1000], max_batch_size=64)
    # r1: no match but above the supermatcher threshold -> not inserted, counts as a match
    # r3: in-batch duplicate of r1 -> a match (NON_MATCH_ID - 1), peer r1
    # r4: unique but skip_persistence -> not inserted, not a match with skip persistence
    # r6: unique -> inserted at the DB's end
    assert r.merged_results == [12, NON_MATCH_ID, 77, NON_MATCH_ID - 1, NON_MATCH_ID, NON_MATCH_ID, 1000]
    assert r.matches == [True, True, True, True, True, True, False]
    assert r.matches_with_skip_persistence == [True, True, True, True, False, True, False]
    assert r.match_ids == [[12, 40], [], [77], [], [], [], []]
    assert r.matched_batch_request_ids == [[], [], [], ["r1"], [], [], []]
    assert r.successful_reauths == [False, False, True, False, False, False, False]
    assert r.full_face_mirror_attack_detected == [False] * 7
    assert r.partial_match_counters_right[1] == 5000
    assert r.reauth_target_indices == {"r2": 77} and r.reauth_or_rule_used == {"r2": False}


def test_normal_pass_after_mirror_pass():
    """The mirror pass runs first; in the normal pass a uniqueness request that
    matched only in the mirrored orientation is flagged as a full-face mirror
    attack and not inserted, and the mirror pass's peers are folded in."""
    mirror_out = _pass(final=[12, NON_MATCH_ID, NON_MATCH_ID, NON_MATCH_ID, NON_MATCH_ID, NON_MATCH_ID, 500],
                       counters=[1, 0, 0, 1, 0, 0, 1],
                       lists=[[12], [], [], [U32_MAX - 0], [], [], [500]])
    mirror = assemble_job_result(BATCH, mirror_out, db_sizes=[1000], max_batch_size=64, orientation="mirror")
    assert mirror.full_face_mirror_attack_detected == [False] * 7
    normal_out = _pass(final=[12, NON_MATCH_ID, 77, NON_MATCH_ID - 1, NON_MATCH_ID, NON_MATCH_ID, NON_MATCH_ID],
                       counters=[1, 0, 1, 1, 0, 0, 0],
                       lists=[[12], [], [77], [U32_MAX - 1], [], [], []])
    r = assemble_job_result(BATCH, normal_out, db_sizes=[1000], max_batch_size=64, previous=mirror)
    # r6: mirror matched 500, normal did not -> attack, and not inserted
    assert r.full_face_mirror_attack_detected == [False, False, False, False, False, False, True]
    assert r.full_face_mirror_match_ids[6] == [500]
    # r1 is now inserted (no match in either orientation), r4 skipped
    assert r.merged_results == [12, 1000, 77, NON_MATCH_ID - 1, NON_MATCH_ID, NON_MATCH_ID, NON_MATCH_ID]
    assert r.matches == [True, False, True, True, True, True, True]
    # r3's peers: r1 (normal pass) then r0 (mirror pass)
    assert r.matched_batch_request_ids[3] == ["r1", "r0"]


def test_insertions_over_gpu_shards():
    """Two GPUs with 500 and 499 entries: insertions are dealt from the smaller
    shard and numbered in the round-robin order."""
    ins = distribute_insertions([3, 5, 6], [500, 499])
    assert ins == [[5], [3, 6]]
    merged = [0] * 8
    m = calculate_insertion_indices(merged, ins, [500, 499], 8)
    assert merged[3] == 999 and merged[5] == 1000 and merged[6] == 1001
    assert [i for i, x in enumerate(m) if not x] == [3, 5, 6]


def test_pass_output_from_batched_results():
    reqs = [Request(code=None, mask=None, n_rot=16, mirrored=True),
            Request(code=None, mask=None, kind="reauth", target=9, mirrored=True),
            Request(code=None, mask=None, n_rot=1)]
    res = [Result(matches=[4, 2], mirror_matches=[8], match_count=300, mirror_match_count=1),
           Result(reauth_match=True, reauth_mirror_match=False), Result()]
    n = pass_output_from_requests(reqs, res)
    assert list(n.final_results) == [2, 9, NON_MATCH_ID]
    assert list(n.match_counters) == [300, 1, 0]
    assert list(n.all_matches[0, :2]) == [2, 4] and n.all_matches[1, 0] == 9
    m = pass_output_from_requests(reqs, res, mirrored=True)
    assert list(m.final_results) == [8, NON_MATCH_ID, NON_MATCH_ID]
    batch = BatchInfo(["a", "b", "c"], ["uniqueness", "reauth", "uniqueness"], reauth_target_indices={"b": 9})
    r = assemble_job_result(batch, n, db_sizes=[100], max_batch_size=8)
    assert r.successful_reauths == [False, True, False]
    assert r.merged_results == [2, 9, 100] and r.matches == [True, True, False]


def test_reauth_without_target_is_refused():
    import pytest
    batch = BatchInfo(["a"], ["reauth"])
    out = _pass(final=[NON_MATCH_ID], counters=[0], lists=[[]])
    with pytest.raises(ValueError, match="no target"):
        assemble_job_result(batch, out, db_sizes=[10], max_batch_size=8)
