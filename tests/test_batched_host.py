"""Host-side logic of the batched launch (no GPU): the row descriptors that
point variants at shared base queries with the mirror bit, and the
expansion rule the device applies to them (rotation of the mirrored share)
checked against the oracle's mirror_share / rotate_share."""
from __future__ import annotations

import numpy as np

from oracle import oracle
from irisb200.batched import attach_bases, centred_rotations, pack


def expand_row(base: np.ndarray, d: int) -> np.ndarray:
    """The row that expand_rows_kernel builds for descriptor d from the base
    queries `base` [n][K], restated with numpy (4-coefficient columns)."""
    K = base.shape[1]
    src, rot, mirror = d >> 8, d & 0x7F, bool(d & 0x80)
    left = 15 - rot
    cols = base[src].reshape(K // 800, 200, 4).astype(np.int64)
    src_col = (np.arange(200) + left) % 200
    if mirror:
        src_col = np.where(src_col < 100, 99 - src_col, 299 - src_col)
    out = cols[:, src_col, :]
    if mirror and K == 12800:
        out[8:] = -out[8:]
    return (out % 65536).astype(np.uint16).reshape(K)


def test_attach_bases_sets_source_and_mirror_bit():
    variants = [list(centred_rotations(n)) for n in (31, 31, 16, 1, 1)]
    base_of = [0, 0, 1, 2, 2]
    mirrored = [False, True, False, False, True]
    lay = pack(variants)
    out = attach_bases(lay, base_of, mirrored)
    assert (lay.row_desc == out.row_desc).sum() == (lay.row_desc == 0xFFFFFFFF).sum() + \
        sum(len(r) for v, r in enumerate(variants) if base_of[v] == v and not mirrored[v])
    for r, d in enumerate(lay.row_desc):
        if d == 0xFFFFFFFF:
            assert out.row_desc[r] == 0xFFFFFFFF
            continue
        v = int(d) >> 8
        e = int(out.row_desc[r])
        assert e >> 8 == base_of[v]
        assert bool(e & 0x80) == mirrored[v]
        assert e & 0x7F == int(d) & 0xFF
    assert np.array_equal(out.seg_query, lay.seg_query) and np.array_equal(out.seg_mask, lay.seg_mask)


def test_device_mirror_rule_matches_oracle():
    rng = np.random.default_rng(11)
    for K, flip in ((12800, True), (6400, False)):
        base = rng.integers(0, 65536, (2, K), dtype=np.uint16)
        mirrored = oracle.mirror_share(base[1], flip)
        for rot in range(31):
            assert np.array_equal(expand_row(base, (1 << 8) | 0x80 | rot), oracle.rotate_share(mirrored, rot))
            assert np.array_equal(expand_row(base, (0 << 8) | rot), oracle.rotate_share(base[0], rot))
