"""Host-side share encoding of the library (irs_encode_iris) against the
oracle's encode_iris_code / encode_mask_code / preprocess (no GPU), and the
deletion record (the default iris: all-zero code, full mask)."""
from __future__ import annotations

import numpy as np

import irisb200


def test_encode_iris_matches_oracle(oracle):
    rng = np.random.default_rng(11)
    for seed in (0, 1, 123456789):
        code = rng.integers(0, 2 ** 63, 200, dtype=np.int64).astype(np.uint64)
        mask = rng.integers(0, 2 ** 63, 200, dtype=np.int64).astype(np.uint64)
        c, m = irisb200.encode_iris(code, mask, seed)
        assert np.array_equal(c, oracle.encode_iris_code(code, mask, seed))
        assert np.array_equal(m, oracle.encode_mask_code(mask, seed))
        cq, mq = irisb200.encode_iris(code, mask, seed, preprocess=True)
        for p in range(3):
            assert np.array_equal(cq[p], oracle.preprocess_query(p, c[p]))
            assert np.array_equal(mq[p], oracle.preprocess_query(p, m[p]))


def test_deletion_record(oracle):
    c, m = irisb200.deletion_record()
    zeros, ones = np.zeros(200, np.uint64), np.full(200, 0xFFFFFFFFFFFFFFFF, np.uint64)
    assert np.array_equal(c, oracle.encode_iris_code(zeros, ones, 0))
    assert np.array_equal(m, oracle.encode_mask_code(ones, 0))
