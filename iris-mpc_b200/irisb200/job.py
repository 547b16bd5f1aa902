"""Per-batch result record of the server actor (ServerJobResult).

The reference's actor turns the device outputs of one batch into a
ServerJobResult (iris-mpc-common/src/job.rs:365-437) in
iris-mpc-gpu/src/server/actor.rs:1159-1520 (after the protocol) and
1679-1712 (the record): per request the merged first match, whether the
request is treated as a match or inserted as a new unique entry (and at which
index), the matched DB ids, the per-eye partial matches with their counters
and rotation indices, the batch peers a request matched, the reauth outcome
and the full-face mirror attack flag built from the mirror orientation's pass.

`assemble_job_result` does the same from this library's outputs: the
reference-layout final results, match counters and match ids of the two-eye
merge (DistanceComparator.fetch_final_results), optionally the per-eye
partial matches (SubsetPass / per-eye comparators) and the previous
orientation's record.  `pass_output_from_requests` builds that input from the
per-request results of BatchedEngine / ContinuousServer.  Service fields that
do not come from the hot path (SQS sequence numbers, metadata, iris shares for
storage, modifications, identity updates) are left to the caller.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

NON_MATCH_ID = 0xFFFFFFFF
U32_MAX = 0xFFFFFFFF
SUPERMATCH_THRESHOLD = 4000  # iris-mpc-gpu/src/server/actor.rs:117
MAX_MATCHES_LEN = 256
UNIQUENESS = "uniqueness"
REAUTH = "reauth"
RESET_CHECK = "reset_check"


@dataclass
class BatchInfo:
    """The request-level fields of a BatchQuery the record carries over."""
    request_ids: list
    request_types: list
    skip_persistence: list | None = None
    reauth_target_indices: dict = field(default_factory=dict)  # request id -> DB index
    reauth_use_or_rule: dict = field(default_factory=dict)     # request id -> bool
    deletion_indices: list = field(default_factory=list)

    def __post_init__(self):
        n = len(self.request_ids)
        if len(self.request_types) != n:
            raise ValueError("request_ids and request_types differ in length")
        if self.skip_persistence is None:
            self.skip_persistence = [False] * n
        if len(self.skip_persistence) != n:
            raise ValueError("skip_persistence has the wrong length")


@dataclass
class PassOutput:
    """Device outputs of one orientation's pass over the batch.

    final_results / match_counters / all_matches: the two-eye merge in the
    reference layout (fetch_final_results / fetch_match_counters /
    fetch_all_match_ids): smallest matched DB id, NON_MATCH_ID, or
    NON_MATCH_ID - 1 for a request that matched an earlier one of its batch;
    match ids hold DB ids and U32_MAX - j for batch request j.
    partial_*: per-eye matches (ids, untruncated counters, and per id the
    matching rotation indices), or None when the pass did not collect them."""
    final_results: np.ndarray
    match_counters: np.ndarray
    all_matches: np.ndarray
    partial_ids_left: list | None = None
    partial_ids_right: list | None = None
    partial_counters_left: list | None = None
    partial_counters_right: list | None = None
    partial_rotations_left: list | None = None
    partial_rotations_right: list | None = None


@dataclass
class ServerJobResult:
    """The hot-path fields of ServerJobResult (iris-mpc-common/src/job.rs:365-437)."""
    merged_results: list
    request_ids: list
    request_types: list
    matches: list
    matches_with_skip_persistence: list
    skip_persistence: list
    match_ids: list
    full_face_mirror_match_ids: list
    partial_match_ids_left: list
    partial_match_ids_right: list
    partial_match_rotation_indices_left: list
    partial_match_rotation_indices_right: list
    full_face_mirror_partial_match_ids_left: list
    full_face_mirror_partial_match_ids_right: list
    partial_match_counters_left: list
    partial_match_counters_right: list
    full_face_mirror_partial_match_counters_left: list
    full_face_mirror_partial_match_counters_right: list
    deleted_ids: list
    matched_batch_request_ids: list
    successful_reauths: list
    reauth_target_indices: dict
    reauth_or_rule_used: dict
    full_face_mirror_attack_detected: list


def distribute_insertions(results, db_sizes) -> list:
    """distribute_insertions (actor.rs:3197-3210): insertion request indices
    dealt round-robin to the devices, starting at the first device with the
    smallest DB."""
    ret = [[] for _ in db_sizes]
    c = list(db_sizes).index(min(db_sizes))
    for r in results:
        ret[c].append(r)
        c = (c + 1) % len(db_sizes)
    return ret


def calculate_insertion_indices(merged_results: list, insertion_list, db_sizes, batch_size: int) -> list:
    """calculate_insertion_indices (actor.rs:3270-3303): the k-th insertion,
    taken round-robin over the devices' lists starting at the device that holds
    the earliest request, gets global index sum(db_sizes) + k and is marked
    not-a-match.  Returns `matches` (True except for the insertions);
    merged_results is updated in place."""
    matches = [True] * batch_size
    last = sum(db_sizes)
    min_index, min_val = 0, None
    for i, lst in enumerate(insertion_list):
        if lst and (min_val is None or lst[0] < min_val):
            min_index, min_val = i, lst[0]
    c = 0
    while True:
        for i in range(len(insertion_list)):
            idx = (i + min_index) % len(insertion_list)
            if c >= len(insertion_list[idx]):
                return matches
            r = insertion_list[idx][c]
            merged_results[r] = last
            matches[r] = False
            last += 1
        c += 1


def assemble_job_result(batch: BatchInfo, out: PassOutput, db_sizes, max_batch_size: int,
                        orientation: str = "normal", previous: ServerJobResult | None = None) -> ServerJobResult:
    """The actor's record of one orientation's pass (actor.rs:1159-1520,
    1679-1712).  db_sizes: the DB length of each GPU shard before the batch
    (one entry per GPU).  previous: the mirror orientation's record when this
    is the normal pass of a mirror-checked batch (the mirror pass runs first).
    Does not write the DB; the insertion indices it assigns are where the
    caller appends the new entries."""
    if orientation not in ("normal", "mirror"):
        raise ValueError("orientation is 'normal' or 'mirror'")
    n = len(batch.request_ids)
    final = [int(x) for x in np.asarray(out.final_results)[:n]]
    counters = [int(x) for x in np.asarray(out.match_counters)[:n]]
    am = np.asarray(out.all_matches)
    match_ids = [[int(x) for x in am[i, :min(counters[i], am.shape[1])]] for i in range(n)]

    def per_query(lst, default):
        return [list(x) for x in lst[:n]] if lst is not None else [list(default) for _ in range(n)]

    pl_ids = per_query(out.partial_ids_left, [])
    pr_ids = per_query(out.partial_ids_right, [])
    pl_cnt = [int(x) for x in out.partial_counters_left[:n]] if out.partial_counters_left is not None else [0] * n
    pr_cnt = [int(x) for x in out.partial_counters_right[:n]] if out.partial_counters_right is not None else [0] * n
    pl_rot = per_query(out.partial_rotations_left, [])
    pr_rot = per_query(out.partial_rotations_right, [])

    merged = list(final)
    use_prev = orientation == "normal" and previous is not None
    ffm_ids = [[] for _ in range(n)]
    ffm_pl, ffm_pr = [[] for _ in range(n)], [[] for _ in range(n)]
    ffm_cl, ffm_cr = [0] * n, [0] * n
    if use_prev:
        attack = [merged[i] == NON_MATCH_ID and previous.matches_with_skip_persistence[i]
                  and batch.request_types[i] == UNIQUENESS for i in range(n)]
        ffm_ids = [list(x) for x in previous.match_ids]
        ffm_pl = [list(x) for x in previous.partial_match_ids_left]
        ffm_pr = [list(x) for x in previous.partial_match_ids_right]
        ffm_cl = list(previous.partial_match_counters_left)
        ffm_cr = list(previous.partial_match_counters_right)
    else:
        attack = [False] * n

    # uniqueness requests without a match (in either orientation when the
    # mirror pass ran first) and below the supermatcher threshold
    unique = [i for i in range(n)
              if batch.request_types[i] == UNIQUENESS and merged[i] == NON_MATCH_ID
              and pl_cnt[i] <= SUPERMATCH_THRESHOLD and pr_cnt[i] <= SUPERMATCH_THRESHOLD
              and not (use_prev and previous.matches_with_skip_persistence[i])]
    insert = [i for i in unique if not batch.skip_persistence[i]]
    skipped = [i for i in unique if batch.skip_persistence[i]]
    matches = calculate_insertion_indices(merged, distribute_insertions(insert, db_sizes), db_sizes, n)
    matches_skip = list(matches)
    for i in skipped:
        matches_skip[i] = False

    # batch peers: dummy ids U32_MAX - j of earlier batch requests j
    peers = [[batch.request_ids[U32_MAX - x] for x in ids if x > U32_MAX - n] for ids in match_ids]
    if previous is not None:
        for i in range(n):
            for rid in previous.matched_batch_request_ids[i]:
                if rid not in peers[i]:
                    peers[i].append(rid)
    filtered = [[x for x in ids if x <= U32_MAX - max_batch_size] for ids in match_ids]
    for i in range(n):
        if batch.request_types[i] == REAUTH and batch.request_ids[i] not in batch.reauth_target_indices:
            raise ValueError(f"reauth request {batch.request_ids[i]!r} has no target index")
    reauth_ok = [batch.request_types[i] == REAUTH
                 and batch.reauth_target_indices[batch.request_ids[i]] in filtered[i] for i in range(n)]
    return ServerJobResult(
        merged_results=merged, request_ids=list(batch.request_ids), request_types=list(batch.request_types),
        matches=matches, matches_with_skip_persistence=matches_skip, skip_persistence=list(batch.skip_persistence),
        match_ids=filtered, full_face_mirror_match_ids=ffm_ids,
        partial_match_ids_left=pl_ids, partial_match_ids_right=pr_ids,
        partial_match_rotation_indices_left=pl_rot, partial_match_rotation_indices_right=pr_rot,
        full_face_mirror_partial_match_ids_left=ffm_pl, full_face_mirror_partial_match_ids_right=ffm_pr,
        partial_match_counters_left=pl_cnt, partial_match_counters_right=pr_cnt,
        full_face_mirror_partial_match_counters_left=ffm_cl, full_face_mirror_partial_match_counters_right=ffm_cr,
        deleted_ids=list(batch.deletion_indices), matched_batch_request_ids=peers,
        successful_reauths=reauth_ok, reauth_target_indices=dict(batch.reauth_target_indices),
        reauth_or_rule_used=dict(batch.reauth_use_or_rule), full_face_mirror_attack_detected=attack)


def pass_output_from_requests(requests, results, mirrored: bool = False) -> PassOutput:
    """PassOutput of one orientation from BatchedEngine / ContinuousServer
    results (irisb200.batched.Result per request): a uniqueness request's
    sorted DB matches (of its mirrored variant when `mirrored`), a reauth
    request's match bit against its target (the reference scans reauth
    queries against the whole DB and checks the target's id among the
    matches, actor.rs:1463-1475; the batched path compares with the target
    alone).  A request without a variant in this orientation has no match.
    The batched paths do not compare a batch with itself, so no batch peers
    appear; counters are the list lengths unless the result carries the
    untruncated count."""
    n = len(requests)
    final = np.full(n, NON_MATCH_ID, np.uint32)
    counters = np.zeros(n, np.uint32)
    am = np.zeros((n, MAX_MATCHES_LEN), np.uint32)
    for i, (r, res) in enumerate(zip(requests, results)):
        if r.kind == REAUTH:
            hit = res.reauth_mirror_match if mirrored else res.reauth_match
            ids = [int(r.target)] if hit else []
            count = len(ids)
        else:
            ids = list(res.mirror_matches if mirrored else res.matches)
            count = getattr(res, "mirror_match_count" if mirrored else "match_count", None)
            count = len(ids) if count is None else int(count)
        if ids:
            final[i] = min(ids)
            am[i, :min(len(ids), MAX_MATCHES_LEN)] = sorted(ids)[:MAX_MATCHES_LEN]
        counters[i] = count
    return PassOutput(final, counters, am)
