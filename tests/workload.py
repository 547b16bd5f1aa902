"""Seeded synthetic workload built with the CPU oracle (test infrastructure).

Irises: code bits uniform, mask kept per real/imaginary pair with p = 0.9.
A fraction of the queries are planted near-duplicates of a DB entry (code bits
flipped with p = 0.2, rotated by r in [-15, 15]); the rest are fresh irises.
Shares follow the degree-1 GR4 Shamir encoding of the oracle; the DB-side
share seed of entry e is rng64(db_seed ^ 0x5EED, e), which is also the
definition the device-side synthetic DB generator follows.
"""
from __future__ import annotations

import numpy as np

SEEDS = [([0] * 8, [2] * 8), ([1] * 8, [0] * 8), ([2] * 8, [1] * 8)]


def db_share_seed(O, db_seed: int, e: int) -> int:
    return int(O.lib().orc_rng64(db_seed ^ 0x5EED, e))


def make_db(O, n: int, db_seed: int):
    """Returns (codes, masks, code_shares [3][n][12800], mask_shares [3][n][6400])."""
    codes, masks = [], []
    cs = np.zeros((3, n, 12800), np.uint16)
    ms = np.zeros((3, n, 6400), np.uint16)
    for e in range(n):
        c, m = O.iris_random(db_seed, e)
        codes.append(c)
        masks.append(m)
        s = db_share_seed(O, db_seed, e)
        cs[:, e] = O.encode_iris_code(c, m, s)
        ms[:, e] = O.encode_mask_code(m, s)
    return codes, masks, cs, ms


def make_queries(O, n_queries: int, db_codes, db_masks, q_seed: int, planted: dict):
    """planted: {query index: (db entry, rotation in -15..15)}.
    Returns base preprocessed query shares per party: code [3][nq][12800],
    mask [3][nq][6400], plus the plaintext queries."""
    qc = np.zeros((3, n_queries, 12800), np.uint16)
    qm = np.zeros((3, n_queries, 6400), np.uint16)
    plain = []
    for j in range(n_queries):
        if j in planted:
            e, r = planted[j]
            c = O.iris_flip(q_seed, j, 0.2, db_codes[e])
            c = O.iris_rotate(c, r)
            m = O.iris_rotate(db_masks[e], r)
        else:
            c, m = O.iris_random(q_seed ^ 0x9999, j)
        plain.append((c, m))
        s = int(O.lib().orc_rng64(q_seed ^ 0x7777, j))
        sc = O.encode_iris_code(c, m, s)
        sm = O.encode_mask_code(m, s)
        for p in range(3):
            qc[p, j] = O.preprocess_query(p, sc[p])
            qm[p, j] = O.preprocess_query(p, sm[p])
    return qc, qm, plain


def rotated_rows(O, base: np.ndarray) -> np.ndarray:
    """[nq][K] -> [nq*31][K] (query row q*31 + r = rotation r)."""
    return np.stack([O.rotate_share(base[j], r) for j in range(base.shape[0]) for r in range(31)])


def expected_bitmap(O, qc, qm, db_cs, db_ms, threshold_a, n_threads=0):
    nq = qc.shape[1]
    q_code = [rotated_rows(O, qc[p]) for p in range(3)]
    q_mask = [rotated_rows(O, qm[p]) for p in range(3)]
    return O.cpu_plain_match(q_code, q_mask, nq, [db_cs[p] for p in range(3)], [db_ms[p] for p in range(3)],
                             threshold_a, n_threads)


def expected_variant_hits(O, cs, ms, qc, qm, rotations, mirrored, entries, threshold_a):
    """Entries matched by one query variant on the CPU: the per-party dots of
    the variant's rotation rows (indices into all 31 rotations, 15 = centre)
    against DB records `entries`, summed over parties (mask x2), thresholded,
    OR over the rows.  qc [3][12800] / qm [3][6400] are the base query shares."""
    base_c = [O.mirror_share(qc[p], True) if mirrored else qc[p] for p in range(3)]
    base_m = [O.mirror_share(qm[p], False) if mirrored else qm[p] for p in range(3)]
    entries = np.asarray(entries)
    code = 0
    mask = 0
    for p in range(3):
        rc = np.stack([O.rotate_share(base_c[p], r) for r in rotations])
        rm = np.stack([O.rotate_share(base_m[p], r) for r in rotations])
        code = code + O.dot_u16(rc, cs[p][entries]).astype(np.uint64)
        mask = mask + 2 * O.dot_u16(rm, ms[p][entries]).astype(np.uint64)
    hit = O.match_predicate(code % 65536, mask % 65536, threshold_a).max(axis=0)
    return [int(e) for e, h in zip(entries, hit) if h]
