"""OR-policy bitmap and lookback records (actor.rs:3601-3660) on the host,
and their per-shard view (no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from irisb200.policy import generate_luc_records, prepare_or_policy_bitmap, row_words, shard_or_policy_bitmap


def _bits(bm, n):
    return np.unpackbits(bm.view(np.uint8), axis=1, bitorder="little")[:, :n]


def test_prepare_or_policy_bitmap():
    bm = prepare_or_policy_bitmap(700, [[0, 63, 64, 699], [], [5]], 4)
    assert bm.shape == (4, row_words(700)) and row_words(700) == 22
    b = _bits(bm, 700)
    assert b[0].nonzero()[0].tolist() == [0, 63, 64, 699]
    assert b[1].sum() == 0 and b[2].nonzero()[0].tolist() == [5] and b[3].sum() == 0
    with pytest.raises(ValueError):
        prepare_or_policy_bitmap(700, [[700]], 1)


def test_generate_luc_records():
    assert generate_luc_records(100, [[1], [2]], 0, 2) == [[1], [2]]
    assert generate_luc_records(10, [], 3, 2) == [[7, 8, 9, 10], [7, 8, 9, 10]]
    assert generate_luc_records(2, [], 5, 1) == [[0, 1, 2]]  # no underflow
    out = generate_luc_records(10, [[9, 1], [4], [12, 3]], 2, 3, skip_lookback_requests={1})
    assert out == [[1, 8, 9, 10], [4], [3, 8, 9, 10, 12]]


def test_shard_or_policy_bitmap():
    world, n = 3, 1000
    rng = np.random.default_rng(4)
    rules = [sorted(rng.choice(n, 40, replace=False).tolist()) for _ in range(5)]
    glob = prepare_or_policy_bitmap(n, rules, 5)
    for rank in range(world):
        local_n = (n - rank + world - 1) // world
        loc = shard_or_policy_bitmap(glob, n, rank, world, local_n)
        assert loc.shape == (5, row_words(local_n))
        b = _bits(loc, local_n)
        for q in range(5):
            assert [int(x) * world + rank for x in b[q].nonzero()[0]] == [e for e in rules[q] if e % world == rank]
